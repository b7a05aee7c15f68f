// noalloc.cu -- the rigid-lid pressure right-hand side for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or allocator it
// does not own, plug-in hosts that forbid device allocation after start-up, or a step that
// must not change the device's memory footprint. pawsim_pressure_rhs_noalloc gives them the
// right-hand side of the rigid-lid pressure equation (div of the summed layer transports
// over dt, with its mean removed) from device arrays they already hold, without allocating.
// Its only scratch -- the partial sums of the mean -- lives in the file-scope array below,
// which every GPU that loads this library keeps until the process exits.
#include <mutex>

#include "../../include/pawsim_b200.h"
#include "common.cuh"
#include "pressure.cuh"

namespace pawsim {

namespace {

// slot 0: the global sum; slots 1..: one partial sum per 8 grid rows
constexpr int kNoallocScratch = 4096;
__device__ __align__(256) double g_rhs_scratch[kNoallocScratch];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device. In host code the array's name
// is only a host-side stand-in, so the address is looked up once per device, with that
// device current, and cached.
int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= kMaxDevices) return PAWSIM_GPU_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_rhs_scratch);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace

}  // namespace pawsim

extern "C" int pawsim_pressure_rhs_noalloc(const double* u, const double* v, const double* h, int Nx, int Ny,
                                           int Nlay, int pitch, double dx, double dy, double dt, int wall_ew,
                                           int wall_ns, int thick_scheme, int serial_sum, double* rhs,
                                           void* stream) {
  using namespace pawsim;
  if (!u || !v || !h || !rhs) return PAWSIM_GPU_EBADCONFIG;
  if (Nx < 4 || Ny < 4 || Nlay < 1 || pitch < Nx || dx <= 0 || dy <= 0 || dt <= 0)
    return PAWSIM_GPU_EBADCONFIG;
  if (thick_scheme != 0 && thick_scheme != 1) return PAWSIM_GPU_EUNSUPPORTED;
  // one partial per 8 rows plus the sum must fit in the static scratch
  if ((size_t)(Ny + 7) / 8 + 1 > (size_t)kNoallocScratch) return PAWSIM_GPU_EUNSUPPORTED;
  // an error left pending by the caller's earlier, unrelated work is reported as such (and
  // cleared) before anything is launched, so that the check after the launches below sees
  // only this call's own errors
  cudaError_t pending = cudaGetLastError();
  if (pending != cudaSuccess)
    return set_cuda_error(pending, "a CUDA error was pending before pawsim_pressure_rhs_noalloc", __FILE__,
                          __LINE__);
  double* scratch = nullptr;
  int r = scratch_address(&scratch);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Grid2 g;
  g.Nx = Nx; g.Ny = Ny; g.pitch = pitch; g.L = Nlay; g.lstride = (size_t)Ny * pitch;
  g.wall_ew = wall_ew; g.wall_ns = wall_ns; g.dx = dx; g.dy = dy; g.dt = dt; g.thick_scheme = thick_scheme;
  g.rdx = 1.0 / dx; g.rdy = 1.0 / dy; g.rdxdt = 1.0 / (dx * dt); g.rdydt = 1.0 / (dy * dt);
  bool serial = serial_sum == 1 || (serial_sum < 0 && (long long)Nx * Ny <= 65536);
  g_launches += launch_pressure_rhs(g, u, v, h, rhs, s);
  launch_sum(rhs, Nx, Ny, pitch, serial, scratch + 1, scratch, s);
  launch_subtract_mean(rhs, Nx, Ny, pitch, scratch, s);
  g_launches += serial ? 2 : 3;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(e, "pawsim_pressure_rhs_noalloc", __FILE__, __LINE__);
  return 0;
}
