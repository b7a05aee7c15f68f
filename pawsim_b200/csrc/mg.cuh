// mg.cuh -- geometric multigrid for the rigid-lid pressure equation on the GPU.
//
// Same hierarchy, operator, restriction and prolongation as the reference's serial AWSIM
// multigrid (model_code/multigrid.c:196-446, 651-932): levels (N+1)/2 down to 1 x 1,
// Ow = Hw/dx^2 and Os = Hs/dy^2 with wall faces zeroed, 2x2 means (area-weighted for
// uneven pairs) and bilinear prolongation with the wall and corner weights. The smoother
// is red-black Gauss-Seidel (weight `omega_rb`) instead of the reference's in-place
// lexicographic sweep, which has no parallel form; convergence is judged by the
// reference's own test, max |pi - Jacobi(pi)| <= tol (multigrid.c:1123-1156).
// Two precisions: plain FP64 V-cycles on pi, or FP32 V-cycles on the correction inside an
// FP64 defect-correction loop (the residual, the update of pi and the test stay FP64).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace pawsim {

struct CoarseDesc;   // the coarse block's launch descriptor (mg.cu)

struct MGOptions {
  int fp32_cycles = 0;     // 0: FP64 V-cycles, 1: FP32 V-cycles in FP64 defect correction
  int fp32_inner = 1;      // FP32 V-cycles per defect-correction step (each after the first
                           // continues from the correction the previous one left)
  int pre = 1, post = 1;   // red-black sweeps before and after the coarse correction
  double omega_rb = 1.0;   // smoother weight
  int full_mg = 0;         // use_fullMG: nested iteration from the coarsest level
  int tile_shape = -1;     // fused level kernels: -1 autotune per level, 0..3 force a tile shape, 4 strips
  // choose omega_rb on the second solve (the first of a time step; the first is the
  // start-up solve from rest): each candidate solves from the same pi and the weight with
  // the fewest V-cycles is kept (the smallest among ties), so the choice is deterministic
  int omega_auto = 0;
};

// candidate weights of the automatic choice
constexpr double kOmegaCandidates[] = {1.0, 1.05, 1.1, 1.15, 1.2, 1.3};

class MGBatch;

class Multigrid {
  friend class MGBatch;

 public:
  // Hc: host array Nx*Ny (x fastest) of the water-column thickness
  Multigrid(int Nx, int Ny, double Lx, double Ly, bool wall_ew, bool wall_ns, const double* Hc_host,
            const MGOptions& opt, cudaStream_t s);
  ~Multigrid();
  bool ok() const { return ok_; }
  // Solve in place on the fine pi (pitched FP64); returns the V-cycle count.
  // maxres_out receives max |pi - Jacobi(pi)| of the last check.
  int solve(double* pi, int pi_pitch, const double* rhs, int rhs_pitch, double tol, int maxiters,
            double* maxres_out);
  // Solve without a host synchronisation: the V-cycle count and the final stopping measure go
  // to the device slots iters_out / maxres_out. Only after a synchronous solve on the same pi
  // and rhs has built the loop (async_ready); *launches receives the kernels enqueued outside
  // the V-cycle graph (each executed cycle adds body_launches(), counted by the caller). When
  // the stream is being captured, the loop is added to the captured graph as its own
  // conditional node instead of launching the loop graph.
  bool async_ready() const;
  int solve_async(double* pi, const double* rhs, double tol, int maxiters, int* iters_out, double* maxres_out,
                  long long* launches);
  int body_launches() const { return body_launches_[opt_.fp32_cycles ? 1 : 0]; }
  // the weight in use (after the automatic choice, the chosen one)
  double omega() const { return opt_.omega_rb; }
  // one evaluation of the stopping measure (for diagnostics and warm-start decisions)
  double max_residual(const double* pi, int pi_pitch, const double* rhs, int rhs_pitch);
  // the same measure, left on the device: *bits = max |pi - Jacobi(pi)| as an integer bit
  // pattern (zeroed first), enqueued on `s` without a host synchronisation
  void measure_async(const double* pi, const double* rhs, unsigned long long* bits, cudaStream_t s);
  // the measures of two candidate fields in one pass: bits[0] for pa, bits[1] for pb
  void measure2_async(const double* pa, const double* pb, const double* rhs, unsigned long long* bits,
                      cudaStream_t s);
  void set_options(const MGOptions& o) { opt_ = o; }
  const MGOptions& options() const { return opt_; }
  int levels() const { return (int)lv_.size(); }
  cudaStream_t stream() const { return s_; }
  void set_stream(cudaStream_t s) { s_ = s; }

  struct Level {
    int Nx, Ny, pitch;
    bool power2;          // transfer to the next coarser level is exactly 2:1
    double *Ow, *Os, *Osum, *rOsum;     // FP64 operator
    float *Ow32, *Os32, *Osum32, *rOsum32;
    double *e, *rhs, *res;              // FP64 work
    float *e32, *rhs32, *res32;         // FP32 work
    double* tmp = nullptr;              // fused down kernel output / up kernel input
    float* tmp32 = nullptr;
    int shape64 = 0, shape32 = 0;       // tile shape of the fused kernels per precision
    bool tuned64 = false, tuned32 = false;
  };

 private:
  // cont: an FP32 cycle that continues from the current correction instead of zero;
  // root: the level the cycle starts from (-1: the finest; lower levels for the nested
  // iteration of use_fullMG, whose solution lives in that level's e)
  template <typename T> void enqueue_vcycle(cudaStream_t s, unsigned long long* measure_bits, bool cont = false,
                                            int root = -1);
  int solve_once(double* pi, const double* rhs, double tol, int maxiters, double* maxres_out);
  // use_fullMG: the nested iteration below the finest level (multigrid.c:1236-1270), leaving
  // the interpolated coarse solution in the fine pi; returns 0 or -1 on a CUDA error
  int full_mg_start(double tol, int maxiters);
  int nsolves_ = 0;
  bool omega_tuned_ = false;
  // the coarse block's descriptor; root >= 0 (at most ctop_) makes a block whose top is that
  // level, iterated from its current e
  template <typename T> CoarseDesc coarse_desc(void* unit_out, int root = -1) const;
  template <typename T> size_t coarse_smem(int root = -1) const;
  template <typename T> void tabulate_coarse(cudaStream_t s);
  // the coarse block's linear map per precision (FP64, FP32) and the options it was made for
  void* cmat_[2] = {nullptr, nullptr};
  int cmat_pre_[2] = {-1, -1}, cmat_post_[2] = {-1, -1};
  double cmat_omega_[2] = {-1, -1};
  template <typename T> void tune(cudaStream_t s);
  void set_fine(double* pi, const double* rhs);
  int build_graph(int prec);
  int capture_body(int prec, cudaGraph_t body, cudaGraphConditionalHandle h);
  int add_loop_node(int prec);
  int body_launches_[2] = {0, 0};   // kernels per executed V-cycle of each graph body
  struct Graphs;
  bool ok_ = false;
  int Nx_, Ny_;
  bool wew_, wns_;
  MGOptions opt_;
  cudaStream_t s_;
  cudaStream_t cap_ = nullptr;     // stream used only to capture the V-cycle graph
  std::vector<Level> lv_;          // index 0 is the coarsest
  int ctop_ = 0;                   // top level of the single-CTA coarse block
  void* dstate_ = nullptr;         // device loop state (stopping measure, iteration count)
  Graphs* g_ = nullptr;
  double* fine_pi_ = nullptr;
  const double* fine_rhs_ = nullptr;
  double *own_e_ = nullptr, *own_rhs_ = nullptr;
};

// The multigrid solves of several models advanced together (the batched ensemble). Members
// with the same level hierarchy form a group; per V-cycle one launch per level and group runs
// the tiles of every member still iterating (blockIdx.z = member), one launch per group applies
// the tabulated coarse maps, and one conditional loop node repeats the cycle until every member
// meets its own stopping test. A member's cycles are its own solve's kernels on its own arrays
// (the same tile arithmetic in the same order), so its iterates, V-cycle count and stopping
// measure equal those of that member's solve alone.
class MGBatch {
 public:
  // members: solvers whose async_ready() holds, with FP64 cycles, pre = post = 1, no
  // use_fullMG, a tabulated coarse map and every tiled level 2:1 (ok() is false otherwise);
  // tol and maxiters per member; it_out[i] / meas_out[i]: device slots that receive member
  // i's V-cycle count and stopping measure after every cycle
  MGBatch(const std::vector<Multigrid*>& members, const std::vector<double>& tol, const std::vector<int>& maxiters,
          const std::vector<int*>& it_out, const std::vector<double*>& meas_out);
  ~MGBatch();
  bool ok() const { return ok_; }
  // enqueue on s, which is being captured into a graph: the loop reset, then the loop as a
  // conditional node of that graph (its body captured on cap); returns 0 or -1
  int capture(cudaStream_t s, cudaStream_t cap);
  // kernels per executed cycle (every group's level launches and the loop test)
  int body_launches() const { return body_launches_; }

 private:
  struct Group;
  std::vector<Group*> groups_;
  void* loop_ = nullptr;       // per member loop state (device)
  int** it_out_ = nullptr;     // device arrays of the members' report slots
  double** meas_out_ = nullptr;
  int n_ = 0;
  int body_launches_ = 0;
  bool ok_ = false;
};

}  // namespace pawsim
