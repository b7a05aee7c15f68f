// dmg.cuh -- the reference's distributed multigrid (pressureSolver 2) on the GPU.
//
// Same hierarchy, operator, transfers and stopping test as the serial build of
// model_code/pressure.c:916-2176: levels halve while both sides are even and above 8;
// face coefficients Hw, Hs of a coarse level are pair means of the finer level's (west
// faces along y, south faces along x) and Hc is the 2x2 mean; V(3,3) cycles of the weighted
// update x += omega_MG ((sum_f O_f x_f - rhs) / sum_f O_f - x); bilinear correction with the
// 9/16, 3/16, 1/16 weights; on the last level a red-black SOR (SOR_rp, tol, maxiters) from
// faces averaged out of its Hc, mean removed; the mean of pi removed after every cycle; stop
// when the largest update of the cycle (last sweep of each smoothing, every correction)
// is at most tol. The reference sweeps in place in x-then-y order, which has no parallel
// form; here each sweep visits red cells then black cells, so iterates agree with the
// reference's to the solver tolerance rather than bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace pawsim {

class DMG {
 public:
  // true when the grid allows the first 2:1 coarsening (otherwise the reference falls back
  // to the gathered multigrid)
  static bool can_start(int Nx, int Ny);
  // Hc: host Nx*Ny (x fastest) water-column thickness
  DMG(int Nx, int Ny, double Lx, double Ly, bool wall_ew, bool wall_ns, const double* Hc_host, double omega,
      double sor_rp, cudaStream_t s);
  ~DMG();
  bool ok() const { return ok_; }
  // V-cycles on pi (pitched, the model's pressure) for rhs until the cycle's largest update
  // is at most tol; returns the cycle count, *last_update the final measure
  int solve(double* pi, int pitch, const double* rhs, int rhs_pitch, double tol, int maxiters,
            double* last_update);
  void set_stream(cudaStream_t s) { s_ = s; }

  struct Level {
    int Nx, Ny;
    double *x, *rhs, *res, *Ow, *Os, *Hc;   // dense Nx*Ny, x fastest; Ow/Os west/south faces
  };

 private:
  void vcycle(int l, unsigned long long* acc);
  bool ok_ = false;
  int Nx_, Ny_;
  bool wew_, wns_;
  double omega_, sor_rp_, dx0_, dy0_, Lx_, Ly_;
  cudaStream_t s_;
  std::vector<Level> lv_;   // index 0 is the finest
  unsigned long long* acc_ = nullptr;
  double *scratch_ = nullptr, *sum_ = nullptr;
  double tol_ = 0;
  int maxiters_ = 0;
};

}  // namespace pawsim
