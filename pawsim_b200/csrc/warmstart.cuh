// warmstart.cuh -- learned warm start of the rigid-lid pressure solve (no counterpart in
// the reference, whose solvers start from the previous step's pressure).
//
// WarmNet: a 4-level convolutional network (about 212k parameters, bf16 weights with an
// FP32 master copy, FP32 accumulation on the tcgen05 tensor cores) with its own forward,
// backward and Adam kernels. Layers (Cin -> Cout at grid level 0..3, level l = H / 2^l):
//   0: 16->32 L0   1: 32->32 L0   pool   2: 32->64 L1   3: 64->64 L1   pool   4: 64->64 L2
//   pool   5: 64->64 L3   up + skip(4)   6: 64->64 L2   up + skip(3)   7: 64->32 L1
//   up + skip(1)   8: 32->32 L0   9: 32->16 L0 (linear; channel 0 is the output)
// ReLU after every layer but the last, 2x2 mean pooling, nearest-neighbour upsampling added
// to the encoder activation of the same level.
//
// WarmStart: the network's inputs and use inside a time step. On a grid coarsened by a
// power of two F (the largest level of at most 256 x 256), it sees
//   c0 = R(rhs) / s_d,  c1 = R(pi1 - pi2) / s_p,  c2 = (R(pi1) - mean) / s_pp
// (R = F x F mean, pi1 = pi(t-1), pi2 = pi(t-2), s_* the RMS of each field) and predicts
// d = R(pi(t) - (2 pi1 - pi2)) / s_p. The guess is 2 pi1 - pi2 + s_p P(d) with P the
// cell-centred bilinear prolongation. Before the solve the multigrid's own stopping
// measure is evaluated for the guess and for pi1; the solve starts from the guess only
// when its measure is lower, so the guess can save V-cycles but never costs accuracy.
// Training pairs (inputs and targets) are collected on the device after solves.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace pawsim {

class Multigrid;

struct WarmNet {
  static constexpr int NL = 10;
  struct LayerDef { int cin, cout, level, relu; };
  static const LayerDef kLayers[NL];

  WarmNet(int H, int W, int Bmax, unsigned long long seed);
  ~WarmNet();
  bool ok() const { return ok_; }
  int H() const { return H_; }
  int W() const { return W_; }
  int Bmax() const { return Bmax_; }
  size_t param_count() const { return nparam_; }

  // in: (B, H, W, 16) bf16 on the device; output channel 0 in out() (B, H, W, 16) FP32
  int forward(const __nv_bfloat16* in, int B, cudaStream_t s);
  const float* out() const { return out_; }
  // loss = mean over pixels of (out0 - target)^2; gradients of all parameters are
  // recomputed (not accumulated). loss_dev receives the loss (device double).
  int backward(const __nv_bfloat16* in, const float* target, int B, double* loss_dev, cudaStream_t s);
  int adam_step(float lr, cudaStream_t s);
  // flattened parameters, per layer w[Cout][3][3][Cin] then b[Cout] (FP32 master values)
  int get_params(float* host) const;
  int set_params(const float* host);
  int get_grads(float* host) const;
  int* err() const { return err_; }

 private:
  bool ok_ = false;
  int H_, W_, Bmax_;
  size_t nparam_ = 0;
  std::vector<void*> allocs_;
  // parameters and optimiser state, one contiguous FP32 block each
  float *w32_ = nullptr, *m_ = nullptr, *v_ = nullptr, *g_ = nullptr;
  size_t woff_[NL], boff_[NL];
  __nv_bfloat16 *wbf_[NL], *wt_[NL];
  int step_ = 0;
  // activations
  __nv_bfloat16 *A_[NL], *P1_, *P2_, *P3_, *U3_, *U2_, *U1_, *dout_, *gs_;
  float* out_;
  float *G_[NL], *tmp_;
  double* part_;
  int* err_;
  template <typename T> T* alloc(size_t n);
  int refresh_bf16(cudaStream_t s);
};

class WarmStart {
 public:
  // the coarsening factor for an Nx x Ny grid, or 0 when the network cannot run on it
  static int factor(int Nx, int Ny);
  WarmStart(int Nx, int Ny, int pitch, int max_pairs, int batch, unsigned long long seed, cudaStream_t s);
  ~WarmStart();
  bool ok() const { return ok_; }
  WarmNet* net() { return net_; }
  int pairs() const { return npairs_; }
  bool trained() const { return trained_; }
  void set_trained(bool t) { trained_ = t; }

  // Before the solve. pi holds pi(t-1). Saves pi(t-1); with `use` and two steps of
  // history writes the guess into pi, keeping pi(t-1) when the guess's stopping measure is
  // not lower. Returns 1 when the guess was computed (the decision stays on the device).
  int before_solve(double* pi, const double* rhs, Multigrid* mg, bool use, cudaStream_t s);
  // After the solve of `rhs` into pi: stores a training pair when collecting, and rotates
  // the history.
  int after_solve(const double* pi, const double* rhs, bool collect, cudaStream_t s);
  // 1 when the last guess was used, 2 when it was rejected, 0 when none was made (host sync)
  int last_decision(cudaStream_t s);
  // Adam on the collected pairs for `epochs` passes; *loss receives the last epoch's mean
  int train(int epochs, float lr, unsigned long long seed, double* loss, cudaStream_t s);

 private:
  bool ok_ = false;
  int Nx_, Ny_, pitch_, F_, Hc_, Wc_, max_pairs_, batch_;
  int npairs_ = 0, next_ = 0, hist_ = 0;
  bool trained_ = false, guessed_ = false;
  WarmNet* net_ = nullptr;
  std::vector<void*> allocs_;
  double *pi1_, *pi2_;               // pi(t-1), pi(t-2) on the fine grid
  double *cr_, *cd_, *cp_, *ct_;     // coarse fields
  double *part_, *scal_;             // reduction partials and the scales of this step
  __nv_bfloat16 *xin_;               // (Bmax, Hc, Wc, 16) network input
  __nv_bfloat16* rx_;                // replay inputs, 4 channels per pair
  float *rt_, *tgt_;                 // replay targets, batch targets
  int* idx_;                         // batch indices
  unsigned long long* bits_;         // stopping measures of guess and of pi(t-1)
  int* decision_;
  double* loss_;
  template <typename T> T* alloc(size_t n);
  void coarse(const double* rhs, const double* pnew, cudaStream_t s);
};

}  // namespace pawsim
