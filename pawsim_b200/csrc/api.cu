// api.cu -- the model object behind the C ABI of include/pawsim_b200.h.
//
// Owns the resident device fields of one model and sequences the hot path exactly as the
// reference's driver does (model_code/pawsim.c:266-304, 471-492): tendency + AB update
// (integrator.c:138-198), then the rigid-lid correction (pressure.c:2254-2300).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pawsim_b200.h"
#include "common.cuh"
#include "dmg.cuh"
#include "mg.cuh"
#include "pressure.cuh"
#include "warmstart.cuh"
#include "tendency.cuh"
#include "tracer.cuh"

namespace pawsim {

static thread_local char g_err[512] = "";
std::atomic<long long> g_launches{0};

int set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  snprintf(g_err, sizeof(g_err), "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
           cudaGetErrorString(e), what, file, line);
  return PAWSIM_GPU_ECUDA;
}

static int fail(int code, const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}

// first guess 2 pi - prev (linear extrapolation of the last two solutions); prev <- pi
__global__ void extrapolate_kernel(double* pi, double* prev, int Nx, int Ny, int pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  size_t c = (size_t)j * pitch + i;
  const double a = pi[c], b = prev[c];
  pi[c] = 2 * a - b;
  prev[c] = a;
}

// rigid-lid column constraint (pressure.c:525-561) when it is not fused into K-tend
__global__ void thickness_fix_kernel(double* h, const double* Hc, int Nx, int Ny, int pitch, size_t ls, int L) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  size_t c = (size_t)j * pitch + i;
  double tot = 0;
  for (int k = 0; k < L; ++k) tot += h[k * ls + c];
  if (tot == 0) return;
  double err = tot - Hc[c];
  for (int k = 0; k < L; ++k) h[k * ls + c] *= (1 - err / tot);
}

// div_rn against the IEEE division, bit for bit (signed zeros and NaN payloads compared as bits)
__global__ void div_check_kernel(const double* x, size_t n, double d, double r, unsigned long long* bad) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = div_rn(x[i], d, r), b = x[i] / d;
  bool same = __double_as_longlong(a) == __double_as_longlong(b) || (a != a && b != b);
  if (!same) atomicAdd(bad, 1ull);
}

__global__ void hc_kernel(const double* hhs, const double* hhb, double* Hc, int Nx, int Ny, int pitch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= Nx || j >= Ny) return;
  size_t c = (size_t)j * pitch + i;
  Hc[c] = hhs[c] - hhb[c];
}

struct Model {
  pawsim_gpu_config c;
  int Nx, Ny, L, pitch, qpitch;
  size_t lstride, plane;
  double dx, dy, t;
  cudaStream_t s = 0;
  std::vector<void*> allocs;
  double *u[2], *v[2], *h[2];
  int cur = 0;
  // AB history: three tendency buffers per variable; h1 holds the newest stored tendency, h2
  // the one before, h3 is free and receives the next (so a recomputed tile still reads intact
  // history)
  double *fu[3], *fv[3], *fh[3];
  int h1 = 0, h2 = 1, h3 = 2;
  int* tile_list = nullptr;   // tiles listed for the fused kernel's exact pass (tendency.cuh)
  double *dtu, *dtv, *dth, *wdia;
  // running averages (allocated by the first accumulation): 9 per-layer sums (u, v, h, M,
  // hu, hv, huu, hvv, huv), then w_dia on L+1 interfaces, then pi
  double* avg = nullptr;
  // tracer (when use_tracer): state b[2] beside u/v/h, tendency history fb[2], restoring
  double *b[2] = {nullptr, nullptr}, *fb[3] = {nullptr, nullptr, nullptr}, *bRelax = nullptr, *bTime = nullptr;
  double *kappa = nullptr, *fsurf = nullptr;   // diapycnal diffusivity (per layer) and surface flux
  double *hhs, *hhb, *Hc, *omz, *taux, *tauy, *fbx, *fby, *uLid, *vLid;
  double *uRelax, *vRelax, *hRelax, *eRelax, *uTime, *vTime, *eTime, *hTime, *wdff, *nu_u, *nu_v;
  double *pi, *rhs, *work, *scratch, *dsum;
  unsigned long long* slots;
  int* diters;
  // corner shadows of the work arrays' last two fills (x-periodic, y-walled grids with the
  // serial build's corners; nullptr otherwise); corner[corner_cur] holds the latest
  double* corner[2] = {nullptr, nullptr};
  int corner_cur = 0;
  double* dragv = nullptr;    // boundary-layer velocities of the quadratic drags over a fraction depth
  int* nonfinite = nullptr;   // raised by the fused kernel when a new state value is not finite
  int nf_calls = 0;           // steps since the flag was last read (check_nonfinite)
  Operator op;
  double gg[LMAX], geff[LMAX];
  std::vector<double> hhs_host, hhb_host;
  Multigrid* mg = nullptr;
  DMG* dmg = nullptr;        // pressureSolver 2 (nullptr: grid falls back to the gathered MG)
  WarmStart* ws = nullptr;   // learned warm start (nullptr until configured)
  int nn_mode = 0;
  bool thickness_fixed = false;
  bool ready = false;
  bool prev_h = false;       // h[1 - cur] holds the thickness at the start of the last step
  double* ez = nullptr;      // energy-diagnostic scratch (terms or partials) and its size
  size_t ez_elems = 0;
  double* ez_out = nullptr;  // KE, PE, Z[L]
  // budget families (config bit q): [term][layer] planes lstride apart, nullptr when off
  double* bud[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* pi_prev = nullptr;   // solution before the last one (pi_guess = 1)
  int pi_solves = 0;           // multigrid solves completed, for the extrapolated guess
  // asynchronous runs (pawsim_gpu_run): each step's solve report in a device ring (iteration
  // count, final stopping measure), read once at the end of the run
  int* run_iters = nullptr;
  double* run_meas = nullptr;
  int run_cap = 0;
  std::vector<int> last_run_iters;
  // asynchronous saves: two staging slots (device, packed planes) with page-locked host
  // copies, filled by a copy stream; busy until the caller releases the slot
  struct SaveSlot {
    double* dev = nullptr;
    double* host = nullptr;
    cudaEvent_t staged = nullptr, done = nullptr;
    bool busy = false;
  };
  SaveSlot save[2];
  int save_next = 0, device = 0;
  size_t save_planes = 0;
  cudaStream_t copy_s = nullptr;
  std::mutex save_mu;
  std::condition_variable save_cv;
  cudaEvent_t ev0, ev1;

  template <typename T> T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(T));
    allocs.push_back(p);
    return (T*)p;
  }
  ~Model() {
    if (copy_s) cudaStreamSynchronize(copy_s);
    for (SaveSlot& q : save) {
      if (q.host) cudaFreeHost(q.host);
      if (q.staged) cudaEventDestroy(q.staged);
      if (q.done) cudaEventDestroy(q.done);
    }
    if (copy_s) cudaStreamDestroy(copy_s);
    delete ws;
    delete dmg;
    delete mg;
    for (void* p : allocs) cudaFree(p);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  bool serial() const {
    if (c.serial_sums == 1) return true;
    if (c.serial_sums == 0) return false;
    return (long long)Nx * Ny <= 65536;
  }
  Grid2 grid2() const {
    Grid2 g;
    g.Nx = Nx; g.Ny = Ny; g.pitch = pitch; g.L = L; g.lstride = lstride;
    g.wall_ew = c.wall_ew; g.wall_ns = c.wall_ns; g.dx = dx; g.dy = dy; g.dt = c.dt;
    g.thick_scheme = c.thick_scheme;
    g.kt00_sigma = c.KT00_sigma;
    g.rdx = 1.0 / dx; g.rdy = 1.0 / dy;
    g.rdxdt = 1.0 / (dx * c.dt); g.rdydt = 1.0 / (dy * c.dt);
    return g;
  }
};

static void fill_d(double* d, size_t n, double v) {
  std::vector<double> tmp(n, v);
  cudaMemcpy(d, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice);
}

static int create(const pawsim_gpu_config* cfg, Model** out) {
  const pawsim_gpu_config& c = *cfg;
  if (c.Nlay < 1 || c.Nlay > LMAX) return fail(PAWSIM_GPU_EBADCONFIG, "Nlay must be in 1..8");
  if (c.pi_guess < 0 || c.pi_guess > 1) return fail(PAWSIM_GPU_EBADCONFIG, "pi_guess must be 0 or 1");
  if (c.budgets < 0 || c.budgets > 31) return fail(PAWSIM_GPU_EBADCONFIG, "budgets is a mask of five families");
  if (c.use_buoyancy && !c.use_tracer) return fail(PAWSIM_GPU_EBADCONFIG, "useBuoyancy requires useTracer");
  if (c.mg_fp32_inner < 0 || c.mg_fp32_inner > 8) return fail(PAWSIM_GPU_EBADCONFIG, "mg_fp32_inner must be in 0..8");
  if (c.Nx < 4 || c.Ny < 4) return fail(PAWSIM_GPU_EBADCONFIG, "Nx and Ny must be at least 4");
  if (c.Ly <= 0 || c.Lx <= 0 || c.dt <= 0) return fail(PAWSIM_GPU_EBADCONFIG, "Lx, Ly and dt must be positive");
  if (c.ts_scheme < 3 || c.ts_scheme > 5)
    return fail(PAWSIM_GPU_EBADCONFIG, "PAWSIM only supports AB1, AB2 and AB3 time stepping so far");
  if (c.mom_scheme < 0 || c.mom_scheme > 3 || c.thick_scheme < 0 || c.thick_scheme > 3)
    return fail(PAWSIM_GPU_EBADCONFIG, "Unknown or unsupported numerical scheme identifier");
  if (c.tau_nrecs < 1 || c.wdia_nrecs < 1) return fail(PAWSIM_GPU_EBADCONFIG, "record counts must be positive");
  if (c.use_tracer && (c.tracer_scheme < 0 || c.tracer_scheme > 2))
    return fail(PAWSIM_GPU_EBADCONFIG, "Unknown or unsupported numerical scheme identifier");
  if (c.use_tracer && (c.K2 < 0 || c.K4 < 0)) return fail(PAWSIM_GPU_EBADCONFIG, "K2 and K4 must be non-negative");
  if (c.solver < 0 || c.solver > 2) return fail(PAWSIM_GPU_EBADCONFIG, "Unknown pressureSolver identifier");
  if (c.check_nonfinite < 0 || c.fail_on_maxiters < 0 || c.fail_on_maxiters > 1)
    return fail(PAWSIM_GPU_EBADCONFIG, "check_nonfinite must be >= 0 and fail_on_maxiters 0 or 1");
  Model* m = new Model();
  m->c = c;
  m->Nx = c.Nx; m->Ny = c.Ny; m->L = c.Nlay;
  m->pitch = round_up(c.Nx, 32);
  m->qpitch = round_up(c.Nx + 1, 32);
  m->lstride = (size_t)c.Ny * m->pitch;
  m->plane = m->lstride;
  m->dx = c.Lx / c.Nx;
  m->dy = c.Ly / c.Ny;
  m->t = c.tmin;
  cudaEventCreate(&m->ev0);
  cudaEventCreate(&m->ev1);
  size_t Ls = m->L * m->lstride;
  bool ok = true;
  for (int b = 0; b < 2; ++b)
    ok &= (m->u[b] = m->alloc<double>(Ls)) && (m->v[b] = m->alloc<double>(Ls)) && (m->h[b] = m->alloc<double>(Ls));
  for (int b = 0; b < 3; ++b)
    ok &= (m->fu[b] = m->alloc<double>(Ls)) && (m->fv[b] = m->alloc<double>(Ls)) && (m->fh[b] = m->alloc<double>(Ls));
  ok &= (m->tile_list = m->alloc<int>(2 + (size_t)((c.Nx + 31) / 32) * ((c.Ny + 7) / 8))) != nullptr;
  ok &= (m->dtu = m->alloc<double>(Ls)) && (m->dtv = m->alloc<double>(Ls)) && (m->dth = m->alloc<double>(Ls));
  if (c.use_tracer) {
    for (int b = 0; b < 2; ++b) ok &= (m->b[b] = m->alloc<double>(Ls)) != nullptr;
    for (int b = 0; b < 3; ++b) ok &= (m->fb[b] = m->alloc<double>(Ls)) != nullptr;
    ok &= (m->bRelax = m->alloc<double>(Ls)) && (m->bTime = m->alloc<double>(Ls));
    ok &= (m->kappa = m->alloc<double>(Ls)) && (m->fsurf = m->alloc<double>(m->plane));
  }
  ok &= (m->wdia = m->alloc<double>((m->L + 1) * m->lstride)) != nullptr;
  ok &= (m->hhs = m->alloc<double>(m->plane)) && (m->hhb = m->alloc<double>(m->plane)) && (m->Hc = m->alloc<double>(m->plane));
  ok &= (m->omz = m->alloc<double>((size_t)(c.Ny + 1) * m->qpitch)) != nullptr;
  ok &= (m->taux = m->alloc<double>(c.tau_nrecs * m->plane)) && (m->tauy = m->alloc<double>(c.tau_nrecs * m->plane));
  ok &= (m->fbx = m->alloc<double>(m->plane)) && (m->fby = m->alloc<double>(m->plane));
  ok &= (m->uLid = m->alloc<double>(m->plane)) && (m->vLid = m->alloc<double>(m->plane));
  ok &= (m->uRelax = m->alloc<double>(Ls)) && (m->vRelax = m->alloc<double>(Ls)) && (m->hRelax = m->alloc<double>(Ls));
  ok &= (m->eRelax = m->alloc<double>(Ls)) && (m->uTime = m->alloc<double>(Ls)) && (m->vTime = m->alloc<double>(Ls));
  ok &= (m->eTime = m->alloc<double>(Ls)) && (m->hTime = m->alloc<double>(m->plane));
  ok &= (m->wdff = m->alloc<double>((size_t)c.wdia_nrecs * (m->L + 1) * m->lstride)) != nullptr;
  ok &= (m->nu_u = m->alloc<double>(Ls)) && (m->nu_v = m->alloc<double>(Ls));
  ok &= (m->pi = m->alloc<double>(m->plane)) && (m->rhs = m->alloc<double>(m->plane)) && (m->work = m->alloc<double>(m->plane));
  ok &= (m->scratch = m->alloc<double>(reduce_scratch_elems(c.Nx, c.Ny))) != nullptr;
  ok &= (m->dsum = m->alloc<double>(8)) != nullptr;
  ok &= (m->slots = m->alloc<unsigned long long>(2)) != nullptr;
  ok &= (m->diters = m->alloc<int>(1)) != nullptr;
  if (c.check_nonfinite > 0) ok &= (m->nonfinite = m->alloc<int>(1)) != nullptr;
  if ((c.quad_drag > 0 && c.hbbl > 0) || (c.quad_drag_surf > 0 && c.hsml > 0))
    ok &= (m->dragv = m->alloc<double>(4 * m->plane)) != nullptr;
  if (!c.wall_ew && c.wall_ns && !c.mpi_corners)
    for (int q = 0; q < 2; ++q) ok &= (m->corner[q] = m->alloc<double>(corner_elems(c.Nlay))) != nullptr;
  m->op.opitch = round_up(c.Nx + 1, 32);
  ok &= (m->op.Ow = m->alloc<double>((size_t)(c.Ny + 1) * m->op.opitch)) != nullptr;
  ok &= (m->op.Os = m->alloc<double>((size_t)(c.Ny + 1) * m->op.opitch)) != nullptr;
  ok &= (m->op.csor = m->alloc<double>(m->plane)) != nullptr;
  if (!ok) {
    delete m;
    return fail(PAWSIM_GPU_ECUDA, "device allocation failed");
  }
  // defaults of model_code/state.c:968-1006
  for (int k = 0; k < m->L; ++k) {
    fill_d(m->hRelax + k * m->lstride, m->lstride, 1000.0 / m->L);
    fill_d(m->eRelax + k * m->lstride, m->lstride, 1000.0 * k / m->L);
    fill_d(m->uTime + k * m->lstride, m->lstride, -1);
    if (m->bTime) fill_d(m->bTime + k * m->lstride, m->lstride, -1);
    fill_d(m->vTime + k * m->lstride, m->lstride, -1);
    fill_d(m->eTime + k * m->lstride, m->lstride, -1);
    m->gg[k] = 9.81;
  }
  fill_d(m->hTime, m->plane, -1);
  m->hhs_host.assign((size_t)c.Nx * c.Ny, 0.0);
  m->hhb_host.assign((size_t)c.Nx * c.Ny, 0.0);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    delete m;
    return set_cuda_error(e, "create", __FILE__, __LINE__);
  }
  *out = m;
  return 0;
}

// resolve a field name to (device base, rows, cols, pitch, count of k)
struct FieldRef {
  double* base;
  int rows, cols, pitch;
  size_t kstride;
  int nk;
  bool writable;
};

static_assert(AVG_LMAX == LMAX, "the averages kernel holds one column of LMAX layers");

// running-average storage: 10 L + 2 fields, and L more for the tracer
static size_t avg_elems(const Model* m) {
  return (size_t)(10 * m->L + 2 + (m->b[0] ? m->L : 0)) * m->lstride;
}

// index of a per-layer running-average sum inside Model::avg (-1 for other names)
static int avg_slot(const std::string& n) {
  static const char* names[9] = {"U_avg", "V_avg", "H_avg", "M_avg", "HU_avg", "HV_avg", "HUU_avg", "HVV_avg",
                                 "HUV_avg"};
  for (int q = 0; q < 9; ++q)
    if (n == names[q]) return q;
  return -1;
}

// the budget families in config-bit order and their output names (defs.h:217-288)
static const int kBudgetTerms[5] = {BU_NTERMS, BU_NTERMS, BH_NTERMS, BE_NTERMS, BB_NTERMS};
static const char* const kBudgetNames[5][BU_NTERMS] = {
    {"UMom_PVadvection", "UMom_Montgomery", "UMom_KEgradient", "UMom_dhdt", "UMom_viscosity", "UMom_hypervisc",
     "UMom_linBotDrag", "UMom_linSurfDrag", "UMom_quadBotDrag", "UMom_quadSurfDrag", "UMom_windStress",
     "UMom_buoyForce", "UMom_relaxation", "UMom_diapycnal", "UMom_baroForcing", "UMom_diaVisc"},
    {"VMom_PVadvection", "VMom_Montgomery", "VMom_KEgradient", "VMom_dhdt", "VMom_viscosity", "VMom_hypervisc",
     "VMom_linBotDrag", "VMom_linSurfDrag", "VMom_quadBotDrag", "VMom_quadSurfDrag", "VMom_windStress",
     "VMom_buoyForce", "VMom_relaxation", "VMom_diapycnal", "VMom_baroForcing", "VMom_diaVisc"},
    {"Thic_advection", "Thic_relaxation"},
    {"Energy_advection", "Energy_Montgomery", "Energy_windStress", "Energy_linBotDrag", "Energy_linSurfDrag",
     "Energy_quadBotDrag", "Energy_quadSurfDrag", "Energy_viscosity", "Energy_hypervisc", "Energy_diaProd",
     "Energy_diaAdv", "Energy_baroForcing", "Energy_buoyForce", "Energy_relaxation", "Energy_diaVisc"},
    {"Tracer_advection", "Tracer_diaAdv", "Tracer_isoDiff", "Tracer_hyperdiff", "Tracer_diaDiff",
     "Tracer_relaxation"}};

static double* budget_plane(Model* m, const std::string& n) {
  for (int f = 0; f < 5; ++f)
    for (int t = 0; m->bud[f] && t < kBudgetTerms[f]; ++t)
      if (n == kBudgetNames[f][t]) return m->bud[f] + (size_t)t * m->L * m->lstride;
  return nullptr;
}

static bool lookup(Model* m, const std::string& n, FieldRef& f) {
  int L = m->L;
  f = FieldRef{nullptr, m->Ny, m->Nx, m->pitch, m->lstride, 1, true};
  if (n == "u") { f.base = m->u[m->cur]; f.nk = L; }
  else if (n == "v") { f.base = m->v[m->cur]; f.nk = L; }
  else if (n == "h") { f.base = m->h[m->cur]; f.nk = L; }
  else if (n == "b" && m->b[0]) { f.base = m->b[m->cur]; f.nk = L; }
  else if (n == "bRelax" && m->bRelax) { f.base = m->bRelax; f.nk = L; }
  else if (n == "bTime" && m->bTime) { f.base = m->bTime; f.nk = L; }
  else if (n == "kappa_dia" && m->kappa) { f.base = m->kappa; f.nk = L; }
  else if (n == "Fsurf_b" && m->fsurf) f.base = m->fsurf;
  else if (n == "uRelax") { f.base = m->uRelax; f.nk = L; }
  else if (n == "vRelax") { f.base = m->vRelax; f.nk = L; }
  else if (n == "hRelax") { f.base = m->hRelax; f.nk = L; }
  else if (n == "eRelax") { f.base = m->eRelax; f.nk = L; }
  else if (n == "uTime") { f.base = m->uTime; f.nk = L; }
  else if (n == "vTime") { f.base = m->vTime; f.nk = L; }
  else if (n == "eTime") { f.base = m->eTime; f.nk = L; }
  else if (n == "nu_u_dia") { f.base = m->nu_u; f.nk = L; }
  else if (n == "nu_v_dia") { f.base = m->nu_v; f.nk = L; }
  else if (n == "hhs") f.base = m->hhs;
  else if (n == "hhb") f.base = m->hhb;
  else if (n == "uLid") f.base = m->uLid;
  else if (n == "vLid") f.base = m->vLid;
  else if (n == "Fbaro_x") f.base = m->fbx;
  else if (n == "Fbaro_y") f.base = m->fby;
  else if (n == "hTime") f.base = m->hTime;
  else if (n == "taux") { f.base = m->taux; f.nk = m->c.tau_nrecs; }
  else if (n == "tauy") { f.base = m->tauy; f.nk = m->c.tau_nrecs; }
  else if (n == "wdia_ff") { f.base = m->wdff; f.nk = m->c.wdia_nrecs * (L + 1); }
  else if (n == "omegaz") { f.base = m->omz; f.rows = m->Ny + 1; f.cols = m->Nx + 1; f.pitch = m->qpitch;
                            f.kstride = 0; }
  else {
    f.writable = false;
    if (n == "pi") f.base = m->pi;
    else if (n == "pi_rhs") f.base = m->rhs;
    else if (n == "Hc") f.base = m->Hc;
    else if (n == "dt_u") { f.base = m->dtu; f.nk = L; }
    else if (n == "dt_v") { f.base = m->dtv; f.nk = L; }
    else if (n == "dt_h") { f.base = m->dth; f.nk = L; }
    else if (n == "wdia") { f.base = m->wdia; f.nk = L + 1; }
    else if (n == "corner_shadow" && m->corner[0]) {
      // the latest corner shadow: [field u, v, h, b][layer][wall side][row][column] as
      // CORNER_F * L * 2 * CORNER_R rows of CORNER_C values
      f.base = m->corner[m->corner_cur]; f.rows = CORNER_F * L * 2 * CORNER_R; f.cols = CORNER_C; f.pitch = CORNER_C;
    }
    else if (n == "tend_u") { f.base = m->fu[m->h1]; f.nk = L; }
    else if (n == "tend_v") { f.base = m->fv[m->h1]; f.nk = L; }
    else if (n == "tend_h") { f.base = m->fh[m->h1]; f.nk = L; }
    else if (m->avg && avg_slot(n) >= 0) { f.base = m->avg + (size_t)avg_slot(n) * L * m->lstride; f.nk = L; }
    else if (m->avg && n == "W_avg") { f.base = m->avg + (size_t)9 * L * m->lstride; f.nk = L + 1; }
    else if (m->avg && n == "P_avg") f.base = m->avg + (size_t)(10 * L + 1) * m->lstride;
    else if (m->avg && m->b[0] && n == "B_avg") { f.base = m->avg + (size_t)(10 * L + 2) * m->lstride; f.nk = L; }
    else if (double* bp = budget_plane(m, n)) { f.base = bp; f.nk = L; }
    else return false;
  }
  return true;
}

static int set_field(Model* m, const char* name, int k, const double* host, size_t n) {
  std::string nm(name ? name : "");
  if (nm == "gg") {
    if ((int)n != m->L) return fail(PAWSIM_GPU_EBADNAME, "gg needs Nlay values");
    for (int q = 0; q < m->L; ++q) {
      if (host[q] < 0) return fail(PAWSIM_GPU_EBADCONFIG, "gFile may contain only non-negative values");
      m->gg[q] = host[q];
    }
    return 0;
  }
  FieldRef f;
  if (!lookup(m, nm, f) || !f.writable) return fail(PAWSIM_GPU_EBADNAME, "unknown or read-only field name");
  if (k < 0 || k >= f.nk) return fail(PAWSIM_GPU_EBADNAME, "field index out of range");
  if (n != (size_t)f.rows * f.cols) return fail(PAWSIM_GPU_EBADNAME, "wrong element count for field");
  PAWSIM_CUDA_OK(cudaMemcpy2DAsync(f.base + k * f.kstride, f.pitch * sizeof(double), host, f.cols * sizeof(double),
                                   f.cols * sizeof(double), f.rows, cudaMemcpyHostToDevice, m->s));
  if (nm == "h") m->prev_h = false;
  if (nm == "pi") m->pi_solves = 0;
  // the state halo fill (state.c:1052-1057) puts +0 on wall faces of the normal velocity
  if (nm == "u" && m->c.wall_ew)
    PAWSIM_CUDA_OK(cudaMemset2DAsync(f.base + k * f.kstride, f.pitch * sizeof(double), 0, sizeof(double), f.rows, m->s));
  if (nm == "v" && m->c.wall_ns)
    PAWSIM_CUDA_OK(cudaMemsetAsync(f.base + k * f.kstride, 0, f.cols * sizeof(double), m->s));
  if (nm == "hhs" || nm == "hhb") {
    std::vector<double>& dst = nm == "hhs" ? m->hhs_host : m->hhb_host;
    memcpy(dst.data(), host, n * sizeof(double));
    m->ready = false;   // the pressure operator and hierarchy depend on Hc
  }
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  return 0;
}

static int get_field(Model* m, const char* name, int k, double* host, size_t n) {
  std::string nm(name ? name : "");
  if (nm == "gg") {
    if ((int)n != m->L) return fail(PAWSIM_GPU_EBADNAME, "gg needs Nlay values");
    memcpy(host, m->gg, m->L * sizeof(double));
    return 0;
  }
  FieldRef f;
  if (!lookup(m, nm, f)) return fail(PAWSIM_GPU_EBADNAME, "unknown field name");
  if (k < 0 || k >= f.nk) return fail(PAWSIM_GPU_EBADNAME, "field index out of range");
  if (n != (size_t)f.rows * f.cols) return fail(PAWSIM_GPU_EBADNAME, "wrong element count for field");
  PAWSIM_CUDA_OK(cudaMemcpy2DAsync(host, f.cols * sizeof(double), f.base + k * f.kstride, f.pitch * sizeof(double),
                                   f.cols * sizeof(double), f.rows, cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  return 0;
}

static int init(Model* m) {
  for (int f = 0; f < 5; ++f) {
    if (!(m->c.budgets & (1 << f)) || m->bud[f]) continue;
    if (f == 4 && !m->c.use_tracer) continue;   // the tracer family needs a tracer
    m->bud[f] = m->alloc<double>((size_t)kBudgetTerms[f] * m->L * m->lstride);
    if (!m->bud[f]) return fail(PAWSIM_GPU_ECUDA, "budget storage allocation failed");
  }
  // state halo fill of state.c:1052-1057: wall-normal velocity is zero on the wall face
  for (int k = 0; k < m->L; ++k) {
    if (m->c.wall_ew)
      PAWSIM_CUDA_OK(cudaMemset2DAsync(m->u[m->cur] + k * m->lstride, m->pitch * sizeof(double), 0, sizeof(double),
                                       m->Ny, m->s));
    if (m->c.wall_ns)
      PAWSIM_CUDA_OK(cudaMemsetAsync(m->v[m->cur] + k * m->lstride, 0, m->Nx * sizeof(double), m->s));
  }
  m->geff[0] = m->gg[0];
  for (int k = 1; k < m->L; ++k) m->geff[k] = m->geff[k - 1] + m->gg[k];
  dim3 b(32, 8), g((m->Nx + 31) / 32, (m->Ny + 7) / 8);
  hc_kernel<<<g, b, 0, m->s>>>(m->hhs, m->hhb, m->Hc, m->Nx, m->Ny, m->pitch);
  ++g_launches;
  launch_operator(m->grid2(), m->Hc, m->op, m->c.sor_rp, m->s);
  g_launches += 2;
  PAWSIM_CUDA_OK(cudaGetLastError());
  if (m->c.use_rl && m->c.solver != PAWSIM_GPU_SOLVER_SOR) {
    delete m->mg;
    m->mg = nullptr;
    std::vector<double> Hc(m->hhs_host.size());
    for (size_t q = 0; q < Hc.size(); ++q) Hc[q] = m->hhs_host[q] - m->hhb_host[q];
    MGOptions o;
    o.fp32_cycles = m->c.mg_fp32;
    o.fp32_inner = m->c.mg_fp32_inner > 0 ? m->c.mg_fp32_inner : 1;
    o.pre = m->c.mg_pre > 0 ? m->c.mg_pre : 1;
    o.post = m->c.mg_post > 0 ? m->c.mg_post : 1;
    o.omega_rb = m->c.mg_omega > 0 ? m->c.mg_omega : 1.0;
    o.omega_auto = m->c.mg_omega < 0 ? 1 : 0;
    o.full_mg = m->c.use_full_mg;
    o.tile_shape = m->c.mg_tile - 1;
    m->mg = new Multigrid(m->Nx, m->Ny, m->c.Lx, m->c.Ly, m->c.wall_ew, m->c.wall_ns, Hc.data(), o, m->s);
    if (!m->mg->ok()) return fail(PAWSIM_GPU_ECUDA, "multigrid allocation failed");
    delete m->dmg;
    m->dmg = nullptr;
    if (m->c.solver == PAWSIM_GPU_SOLVER_MG_DISTRIBUTED && DMG::can_start(m->Nx, m->Ny)) {
      m->dmg = new DMG(m->Nx, m->Ny, m->c.Lx, m->c.Ly, m->c.wall_ew, m->c.wall_ns, Hc.data(), m->c.omega_mg,
                       m->c.sor_rp, m->s);
      if (!m->dmg->ok()) return fail(PAWSIM_GPU_ECUDA, "distributed multigrid allocation failed");
    }
  }
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  m->ready = true;
  return 0;
}

// wind / wDia record interpolation weights (forcing.c:49-68, restoring.c:56-70)
static void record_weights(int nrecs, double period, double t, int* n0, int* n1, double* w0, double* w1) {
  *n0 = 0; *n1 = 0; *w0 = 1; *w1 = 0;
  if (nrecs > 1 && period > 0) {
    double nflt = (fmod(t, period) / period) * nrecs;
    unsigned nm1 = (unsigned)floor(nflt), np1 = (unsigned)ceil(nflt);
    if (np1 == nm1) np1 = nm1 + 1;
    *n0 = (int)nm1;
    *n1 = (int)(np1 % (unsigned)nrecs);
    *w0 = np1 - nflt;
    *w1 = nflt - nm1;
  }
}

static TendParams base_params(Model* m) {
  TendParams p;
  memset(&p, 0, sizeof(p));
  const pawsim_gpu_config& c = m->c;
  p.Nx = m->Nx; p.Ny = m->Ny; p.L = m->L; p.pitch = m->pitch; p.qpitch = m->qpitch; p.lstride = m->lstride;
  p.wall_ew = c.wall_ew; p.wall_ns = c.wall_ns; p.use_rl = c.use_rl;
  p.dx = m->dx; p.dy = m->dy;
  p.rdx = 1.0 / m->dx; p.rdy = 1.0 / m->dy; p.r24 = 1.0 / 24.0;
  p.u = m->u[m->cur]; p.v = m->v[m->cur]; p.h = m->h[m->cur];
  p.hhb = m->hhb; p.hhs = m->hhs; p.Hc = m->Hc; p.omz = m->omz;
  for (int k = 0; k < m->L; ++k) { p.gg[k] = m->gg[k]; p.geff[k] = m->geff[k]; }
  p.h0 = c.h0;
  p.useA2 = (c.A2 > 0) || (c.A2smag > 0);
  p.useA4 = (c.A4 > 0) || (c.A4smag > 0);
  p.A2 = c.A2;
  p.A4sqrt = sqrt(c.A4);
  p.A4 = c.A4;
  // Smagorinsky factors, as work.c:1587-1592 forms them
  p.use_smag = (c.A2smag > 0 ? 1 : 0) | (c.A4smag > 0 ? 2 : 0);
  {
    const double mdx = fmax(m->dx, m->dy);
    p.A2f = (c.A2smag * fmax(m->dx, m->dy) / 3.14159265358979323846) * (c.A2smag * fmax(m->dx, m->dy) / 3.14159265358979323846);
    p.A4f = (c.A4smag / 3.14159265358979323846) * (c.A4smag / 3.14159265358979323846) * (mdx * mdx * mdx * mdx) / 8;
  }
  p.kt00_sigma = c.KT00_sigma;
  p.quad_drag = c.quad_drag;
  p.quad_drag_surf = c.quad_drag_surf;
  p.wfb = c.wind_feedback ? 0.3 : 0.0;
  p.use_fractions = (c.hsml > 0 || c.hbbl > 0) ? 1 : 0;
  p.hsml = c.hsml; p.hmin_surf = c.hmin_surf; p.hbbl = c.hbbl; p.hmin_bot = c.hmin_bot;
  p.use_wind = c.use_wind; p.use_fbaro = c.use_fbaro;
  int n0, n1;
  record_weights(c.tau_nrecs, c.tau_period, m->t, &n0, &n1, &p.tw0, &p.tw1);
  p.taux0 = m->taux + n0 * m->plane; p.taux1 = m->taux + n1 * m->plane;
  p.tauy0 = m->tauy + n0 * m->plane; p.tauy1 = m->tauy + n1 * m->plane;
  p.fbx = m->fbx; p.fby = m->fby;
  p.lin_drag = c.lin_drag; p.lin_drag_surf = c.lin_drag_surf; p.ocean_surf_drag = c.ocean_surf_drag;
  p.uLid = m->uLid; p.vLid = m->vLid;
  p.use_relax = c.use_relax; p.use_wdia = c.use_wdia; p.use_wdia_file = c.use_wdia_file;
  p.use_diavisc = c.use_diavisc;
  record_weights(c.wdia_nrecs, c.wdia_period, m->t, &n0, &n1, &p.ww0, &p.ww1);
  p.wd0 = m->wdff + (size_t)n0 * (m->L + 1) * m->lstride;
  p.wd1 = m->wdff + (size_t)n1 * (m->L + 1) * m->lstride;
  p.hRelax = m->hRelax; p.eRelax = m->eRelax; p.eTime = m->eTime; p.hTime = m->hTime;
  p.uRelax = m->uRelax; p.vRelax = m->vRelax; p.uTime = m->uTime; p.vTime = m->vTime;
  p.nu_u = m->nu_u; p.nu_v = m->nu_v;
  p.wdia_out = m->wdia;
  p.use_buoy = c.use_buoyancy;
  p.b = c.use_tracer ? m->b[m->cur] : nullptr;
  p.conv_diff = c.conv_diff;
  p.nonfinite = m->nonfinite;
  p.corners = m->corner[0] ? m->corner[m->corner_cur] : nullptr;
  p.dragv = m->dragv;
  p.tile_list = m->tile_list;
  p.drag_bot = (c.quad_drag > 0 && c.hbbl > 0) ? 1 : 0;
  p.drag_surf = (c.quad_drag_surf > 0 && c.hsml > 0) ? 1 : 0;
  return p;
}

// A fill of the work arrays in the reference (pawsim_work_load_state): record its corner
// shadow from state buffer `sb` into the other shadow buffer (the kernels of this fill may
// still read the current one) and make it the latest.
static void corner_fill(Model* m, int sb) {
  if (!m->corner[0]) return;
  const int nx = 1 - m->corner_cur;
  launch_corner_capture(m->grid2(), m->u[sb], m->v[sb], m->h[sb], m->b[0] ? m->b[sb] : nullptr, m->corner[nx], m->s);
  ++g_launches;
  m->corner_cur = nx;
}

// check_nonfinite: every K-th step reads and clears the flag the fused kernel raises
static int check_state_finite(Model* m) {
  if (!m->nonfinite || ++m->nf_calls < m->c.check_nonfinite) return 0;
  m->nf_calls = 0;
  int flag = 0;
  PAWSIM_CUDA_OK(cudaMemcpyAsync(&flag, m->nonfinite, sizeof(int), cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaMemsetAsync(m->nonfinite, 0, sizeof(int), m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  if (flag) {
    char msg[160];
    snprintf(msg, sizeof(msg), "the state became non-finite (NaN or Inf) at or before model time %.9g s", m->t);
    return fail(PAWSIM_GPU_ENONFINITE, msg);
  }
  return 0;
}

// fail_on_maxiters: a rigid-lid solve that stopped at maxiters (the reference's warning case,
// pawsim.c:488-491)
static int check_converged(const Model* m, int iters) {
  if (!m->c.fail_on_maxiters || !m->c.use_rl || iters < m->c.maxiters) return 0;
  char msg[160];
  snprintf(msg, sizeof(msg), "the pressure solve reached maxiters (%d) at model time %.9g s", m->c.maxiters, m->t);
  return fail(PAWSIM_GPU_ENOTCONVERGED, msg);
}

// the plain fused kernel, or its budget build when budgets accumulate or buoyancy couples
static int launch_step_kernel(const Model* m, const TendParams& p) {
  const bool ext = p.use_buoy || p.bud_u || p.bud_v || p.bud_h || p.bud_e || p.bud_b;
  return ext ? launch_tendency_budget(p, m->c.mom_scheme, m->c.thick_scheme, m->s)
             : launch_tendency(p, m->c.mom_scheme, m->c.thick_scheme, m->s);
}

static int tendency_eval(Model* m) {
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  TendParams p = base_params(m);
  p.ab_mode = 0;
  p.fu_out = m->dtu; p.fv_out = m->dtv; p.fh_out = m->dth;
  const int nl = launch_step_kernel(m, p);
  if (nl < 0) return fail(PAWSIM_GPU_EUNSUPPORTED, "scheme combination not available");
  g_launches += nl;   // the drag pre-pass, the fused kernel and its exact pass
  corner_fill(m, m->cur);   // the tendency's load_state and face thickness
  PAWSIM_CUDA_OK(cudaGetLastError());
  return 0;
}

// The fused kernel's parameters of integrator step n (AB coefficients of integrator.c:138-198
// with the AB3 start-up, history slots, output buffers); *shift: the step stores its tendency.
static TendParams step_params(Model* m, unsigned n, bool fuse_fix, bool* shift_out) {
  const pawsim_gpu_config& c = m->c;
  TendParams p = base_params(m);
  double dt = c.dt;
  bool shift = true;
  if (c.ts_scheme == 3 || n == 1) {
    p.ab_mode = 1; p.c0 = dt;
    if (c.ts_scheme == 5) shift = false;   // AB3 start-up keeps no history (integrator.c:169-172)
  } else if (c.ts_scheme == 4 || n == 2) {
    p.ab_mode = 2; p.c0 = 3 * dt / 2; p.c1 = dt / 2;
  } else {
    p.ab_mode = 3; p.c0 = 23 * dt / 12; p.c1 = 4 * dt / 3; p.c2 = 5 * dt / 12;
  }
  const int h1 = m->h1, h2 = m->h2, h3 = m->h3;
  p.f1u = m->fu[h1]; p.f1v = m->fv[h1]; p.f1h = m->fh[h1];
  p.f2u = m->fu[h2]; p.f2v = m->fv[h2]; p.f2h = m->fh[h2];
  p.fu_out = m->fu[h3]; p.fv_out = m->fv[h3]; p.fh_out = m->fh[h3];
  p.write_hist = shift ? 1 : 0;
  int nb = 1 - m->cur;
  p.u_out = m->u[nb]; p.v_out = m->v[nb]; p.h_out = m->h[nb];
  p.fuse_thickness_fix = (fuse_fix && c.use_rl) ? 1 : 0;
  const bool budgets = m->bud[0] || m->bud[1] || m->bud[2] || m->bud[3] || m->bud[4];
  if (budgets) {
    p.dt = dt;
    p.bud_u = m->bud[0]; p.bud_v = m->bud[1]; p.bud_h = m->bud[2]; p.bud_e = m->bud[3]; p.bud_b = m->bud[4];
  }
  *shift_out = shift;
  return p;
}

// The model's bookkeeping after the launches of integrator step (history rotation, state
// buffers, time).
static void step_finish(Model* m, const TendParams& p, bool shift) {
  if (shift) {   // newest <- the buffer just written, the previous newest moves back one slot
    const int h1 = m->h1, h2 = m->h2, h3 = m->h3;
    m->h1 = h3;
    m->h2 = h1;
    m->h3 = h2;
  }
  m->cur = 1 - m->cur;
  m->prev_h = true;
  m->t += m->c.dt;
  m->thickness_fixed = p.fuse_thickness_fix != 0;
}

static int integrator_step(Model* m, unsigned n, bool fuse_fix) {
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  const pawsim_gpu_config& c = m->c;
  bool shift = true;
  const TendParams p = step_params(m, n, fuse_fix, &shift);
  const double dt = c.dt;
  const int h1 = m->h1, h2 = m->h2, h3 = m->h3, nb = 1 - m->cur;
  const int nl = launch_step_kernel(m, p);
  if (nl < 0) return fail(PAWSIM_GPU_EUNSUPPORTED, "scheme combination not available");
  g_launches += nl;   // the drag pre-pass, the fused kernel and its exact pass
  if (c.use_tracer) {
    // the tracer reads the state of the start of the step and the w_dia the tendency
    // kernel just wrote; same AB coefficients and history slots
    TracerParams tp;
    tp.Nx = m->Nx; tp.Ny = m->Ny; tp.L = m->L; tp.pitch = m->pitch; tp.lstride = m->lstride;
    tp.wall_ew = c.wall_ew; tp.wall_ns = c.wall_ns;
    tp.scheme = c.tracer_scheme; tp.thick_scheme = c.thick_scheme; tp.kt00_sigma = c.KT00_sigma;
    tp.dx = m->dx; tp.dy = m->dy; tp.K2 = c.K2; tp.K4 = c.K4;
    tp.rdx = 1.0 / m->dx; tp.rdy = 1.0 / m->dy;
    tp.rdxsq = 1.0 / (m->dx * m->dx); tp.rdysq = 1.0 / (m->dy * m->dy);
    tp.use_wdia = c.use_wdia;
    tp.u = m->u[m->cur]; tp.v = m->v[m->cur]; tp.h = m->h[m->cur]; tp.b = m->b[m->cur];
    tp.bRelax = m->bRelax; tp.bTime = m->bTime; tp.wdia = m->wdia;
    tp.ab_mode = p.ab_mode; tp.c0 = p.c0; tp.c1 = p.c1; tp.c2 = p.c2; tp.write_hist = p.write_hist;
    tp.f1b = m->fb[h1]; tp.f2b = m->fb[h2]; tp.fb_out = m->fb[h3]; tp.b_out = m->b[nb];
    tp.bud_b = m->bud[4]; tp.dt = dt;
    tp.use_buoy = c.use_buoyancy;
    for (int k = 0; k < m->L; ++k) tp.gg[k] = m->gg[k];
    tp.use_diadiff = c.use_diadiff; tp.kappa = m->kappa; tp.fsurf = m->fsurf; tp.conv_diff = c.conv_diff;
    tp.corners = p.corners;
    launch_tracer(tp, m->s);
    ++g_launches;
  }
  corner_fill(m, m->cur);   // the tendency's load_state and face thickness (state of the step start)
  PAWSIM_CUDA_OK(cudaGetLastError());
  step_finish(m, p, shift);
  return 0;
}

static int finish_norms(Model* m, const double* field, double* mx, double* rms) {
  launch_norms(field, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
  g_launches += 3;
  double hbuf[2];
  PAWSIM_CUDA_OK(cudaMemcpyAsync(hbuf, m->dsum, 2 * sizeof(double), cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  *mx = hbuf[0];
  *rms = sqrt(hbuf[1] / ((double)m->Nx * (double)m->Ny));
  return 0;
}

static int pressure_correct(Model* m, int update_diags, pawsim_gpu_stats* st) {
  pawsim_gpu_stats local;
  memset(&local, 0, sizeof(local));
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  if (!m->c.use_rl) {
    if (st) *st = local;
    return 0;
  }
  const int cur = m->cur;
  Grid2 g = m->grid2();
  dim3 b(32, 8), gr((m->Nx + 31) / 32, (m->Ny + 7) / 8);
  if (!m->thickness_fixed) {
    thickness_fix_kernel<<<gr, b, 0, m->s>>>(m->h[cur], m->Hc, m->Nx, m->Ny, m->pitch, m->lstride, m->L);
    ++g_launches;
  }
  m->thickness_fixed = false;
  g_launches += launch_pressure_rhs(g, m->u[cur], m->v[cur], m->h[cur], m->rhs, m->s);
  corner_fill(m, cur);   // build_rhs reloads the corrected state (pressure.c:570-606)
  launch_sum(m->rhs, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
  launch_subtract_mean(m->rhs, m->Nx, m->Ny, m->pitch, m->dsum, m->s);
  g_launches += m->serial() ? 2 : 3;
  PAWSIM_CUDA_OK(cudaGetLastError());
  PAWSIM_CUDA_OK(cudaEventRecord(m->ev0, m->s));
  if (m->c.pi_guess == 1 && m->c.solver != PAWSIM_GPU_SOLVER_SOR) {
    // pi holds the last solution; from the third solve on start from the extrapolation
    if (!m->pi_prev) {
      m->pi_prev = m->alloc<double>((size_t)m->Ny * m->pitch);
      if (!m->pi_prev) return fail(PAWSIM_GPU_ECUDA, "pressure history allocation failed");
    }
    if (m->pi_solves >= 2) {
      extrapolate_kernel<<<gr, b, 0, m->s>>>(m->pi, m->pi_prev, m->Nx, m->Ny, m->pitch);
      ++g_launches;
    } else if (m->pi_solves == 1) {
      PAWSIM_CUDA_OK(cudaMemcpyAsync(m->pi_prev, m->pi, (size_t)m->Ny * m->pitch * sizeof(double),
                                     cudaMemcpyDeviceToDevice, m->s));
    }
    ++m->pi_solves;
  }
  int iters = 0;
  if (m->c.solver == PAWSIM_GPU_SOLVER_SOR) {
    if (launch_sor(g, m->pi, m->rhs, m->op, m->c.sor_rp, m->c.pi_tol, m->c.maxiters, m->slots, m->diters, m->s) != 0)
      return fail(PAWSIM_GPU_ECUDA, "cooperative SOR launch failed");
    ++g_launches;
    launch_sum(m->pi, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
    launch_subtract_mean(m->pi, m->Nx, m->Ny, m->pitch, m->dsum, m->s);
    g_launches += m->serial() ? 2 : 3;
    PAWSIM_CUDA_OK(cudaMemcpyAsync(&iters, m->diters, sizeof(int), cudaMemcpyDeviceToHost, m->s));
    PAWSIM_CUDA_OK(cudaEventRecord(m->ev1, m->s));
    PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  } else if (m->c.solver == PAWSIM_GPU_SOLVER_MG) {
    double mres = 0;
    if (m->ws && m->ws->before_solve(m->pi, m->rhs, m->mg, (m->nn_mode & 2) != 0, m->s) < 0)
      return fail(PAWSIM_GPU_ECUDA, "warm-start guess failed");
    iters = m->mg->solve(m->pi, m->pitch, m->rhs, m->pitch, m->c.pi_tol, m->c.maxiters, &mres);
    if (iters < 0) return fail(PAWSIM_GPU_ECUDA, "multigrid solve failed (graph build or stream error)");
    local.stop_measure = mres;
    local.mg_omega = m->mg->omega();
    PAWSIM_CUDA_OK(cudaEventRecord(m->ev1, m->s));
    PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
    if (m->ws) {
      local.warm_start = m->ws->last_decision(m->s);
      if (m->ws->after_solve(m->pi, m->rhs, (m->nn_mode & 1) != 0, m->s) < 0)
        return fail(PAWSIM_GPU_ECUDA, "warm-start pair collection failed");
    }
  } else if (m->dmg) {
    double mu = 0;
    iters = m->dmg->solve(m->pi, m->pitch, m->rhs, m->pitch, m->c.pi_tol, m->c.maxiters, &mu);
    if (iters < 0) return fail(PAWSIM_GPU_ECUDA, "distributed multigrid solve failed");
    // the reference removes the mean of pi once more after copying it back (pressure.c:2169)
    launch_sum(m->pi, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
    launch_subtract_mean(m->pi, m->Nx, m->Ny, m->pitch, m->dsum, m->s);
    g_launches += m->serial() ? 2 : 3;
    local.stop_measure = mu;
    PAWSIM_CUDA_OK(cudaEventRecord(m->ev1, m->s));
    PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  } else {
    // grids without a first clean 2:1 coarsening use the gathered multigrid (pressure.c:2136-2148)
    double mres = 0;
    iters = m->mg->solve(m->pi, m->pitch, m->rhs, m->pitch, m->c.pi_tol, m->c.maxiters, &mres);
    if (iters < 0) return fail(PAWSIM_GPU_ECUDA, "multigrid solve failed (graph build or stream error)");
    local.stop_measure = mres;
    local.mg_omega = m->mg->omega();
    local.fallback = 1;
    PAWSIM_CUDA_OK(cudaEventRecord(m->ev1, m->s));
    PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, m->ev0, m->ev1);
  local.solve_ms = ms;
  local.iters = iters;
  PAWSIM_CUDA_OK(cudaGetLastError());
  if (m->c.pressure_timing) {
    launch_residual_field(g, m->pi, m->rhs, m->op, m->work, m->s);
    ++g_launches;
    int r = finish_norms(m, m->work, &local.residual_max, &local.residual_rms);
    if (r) return r;
  }
  if (update_diags && (m->bud[0] || m->bud[1] || m->bud[3]))
    launch_projection_budget(g, m->pi, m->u[cur], m->v[cur], m->h[cur], m->bud[0], m->bud[1], m->bud[3], m->s);
  else
    launch_projection(g, m->pi, m->u[cur], m->v[cur], m->s);
  ++g_launches;
  if (m->c.pressure_timing) {
    corner_fill(m, cur);   // the divergence norms reload the projected state (pressure.c:693-737)
    g_launches += launch_divergence_field(g, m->u[cur], m->v[cur], m->h[cur], m->work, m->s);
    int r = finish_norms(m, m->work, &local.div_max, &local.div_rms);
    if (r) return r;
  }
  PAWSIM_CUDA_OK(cudaGetLastError());
  if (st) *st = local;
  return iters;
}

// the device ring of per-step solve reports holds at least nsteps entries
static bool ensure_run_ring(Model* m, unsigned nsteps) {
  if ((int)nsteps <= m->run_cap) return true;
  int* ri = m->alloc<int>(nsteps);
  double* rm = m->alloc<double>(nsteps);
  if (!ri || !rm) return false;
  m->run_iters = ri;
  m->run_meas = rm;
  m->run_cap = (int)nsteps;
  return true;
}

// Can the rigid-lid correction run without a host synchronisation? (no report the host must
// form: pressure timing, warm start, the distributed multigrid's host loop, full multigrid)
static bool async_correct_ok(const Model* m) {
  const pawsim_gpu_config& c = m->c;
  if (!c.use_rl) return true;
  if (c.pressure_timing || (m->ws && m->nn_mode)) return false;
  if (c.solver == PAWSIM_GPU_SOLVER_SOR) return true;
  if (c.solver == PAWSIM_GPU_SOLVER_MG) return m->mg && m->mg->async_ready();
  return false;
}

// The rigid-lid correction of pressure_correct without a host synchronisation; the solve's
// iteration count and stopping measure go to the device slots it_out / meas_out (0 without
// the rigid lid).
// The steps of the rigid-lid correction before the solve: thickness constraint (unless the
// fused step applied it), right-hand side with its corner fill, mean removal, and for the
// multigrid the extrapolated first guess (pi_guess = 1).
static int pressure_pre_solve(Model* m) {
  const int cur = m->cur;
  Grid2 g = m->grid2();
  dim3 b(32, 8), gr((m->Nx + 31) / 32, (m->Ny + 7) / 8);
  if (!m->thickness_fixed) {
    thickness_fix_kernel<<<gr, b, 0, m->s>>>(m->h[cur], m->Hc, m->Nx, m->Ny, m->pitch, m->lstride, m->L);
    ++g_launches;
  }
  m->thickness_fixed = false;
  g_launches += launch_pressure_rhs(g, m->u[cur], m->v[cur], m->h[cur], m->rhs, m->s);
  corner_fill(m, cur);
  launch_sum(m->rhs, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
  launch_subtract_mean(m->rhs, m->Nx, m->Ny, m->pitch, m->dsum, m->s);
  g_launches += m->serial() ? 2 : 3;
  if (m->c.solver != PAWSIM_GPU_SOLVER_SOR && m->c.pi_guess == 1) {
    if (m->pi_solves >= 2) {
      extrapolate_kernel<<<gr, b, 0, m->s>>>(m->pi, m->pi_prev, m->Nx, m->Ny, m->pitch);
      ++g_launches;
    } else if (m->pi_solves == 1) {
      PAWSIM_CUDA_OK(cudaMemcpyAsync(m->pi_prev, m->pi, (size_t)m->Ny * m->pitch * sizeof(double),
                                     cudaMemcpyDeviceToDevice, m->s));
    }
    ++m->pi_solves;
  }
  return 0;
}

static int pressure_post_solve(Model* m) {
  launch_projection(m->grid2(), m->pi, m->u[m->cur], m->v[m->cur], m->s);
  ++g_launches;
  PAWSIM_CUDA_OK(cudaGetLastError());
  return 0;
}

static int pressure_correct_async(Model* m, int* it_out, double* meas_out) {
  if (!m->c.use_rl) {
    PAWSIM_CUDA_OK(cudaMemsetAsync(it_out, 0, sizeof(int), m->s));
    return 0;
  }
  int rc = pressure_pre_solve(m);
  if (rc) return rc;
  if (m->c.solver == PAWSIM_GPU_SOLVER_SOR) {
    Grid2 g = m->grid2();
    if (launch_sor(g, m->pi, m->rhs, m->op, m->c.sor_rp, m->c.pi_tol, m->c.maxiters, m->slots, m->diters, m->s) != 0)
      return fail(PAWSIM_GPU_ECUDA, "cooperative SOR launch failed");
    ++g_launches;
    launch_sum(m->pi, m->Nx, m->Ny, m->pitch, m->serial(), m->scratch, m->dsum, m->s);
    launch_subtract_mean(m->pi, m->Nx, m->Ny, m->pitch, m->dsum, m->s);
    g_launches += m->serial() ? 2 : 3;
    PAWSIM_CUDA_OK(cudaMemcpyAsync(it_out, m->diters, sizeof(int), cudaMemcpyDeviceToDevice, m->s));
  } else {
    long long nl = 0;
    if (m->mg->solve_async(m->pi, m->rhs, m->c.pi_tol, m->c.maxiters, it_out, meas_out, &nl) != 0)
      return fail(PAWSIM_GPU_ECUDA, "asynchronous multigrid solve failed");
    g_launches += nl;
  }
  return pressure_post_solve(m);
}

// A batched ensemble of models (no reference counterpart: the reference runs one model per
// process, its multigrid state being file-scope globals, multigrid.c:54-63). Each step the
// fused kernel of every member runs in one launch over a work-list of all members' tiles,
// then each member's rigid-lid correction on its own stream; no host synchronisation. Once
// every member's step has a fixed form (AB3 history shifting, the multigrid loop built), the
// whole step -- the batched launch, and per member the correction with its V-cycle loop as a
// conditional node -- is captured into one CUDA graph per arrangement of the members' state
// buffers (they rotate with period 6) and replayed with one launch per step.
struct EnsGraph {
  std::vector<int> key;               // per member: cur, h1, h2, h3, corner_cur
  cudaGraphExec_t exec = nullptr;
  TendParams* d_params = nullptr;     // the parameter blocks the graph's batched launch reads
  std::vector<TendParams> h_params;   // what d_params holds
  long long launches = 0;             // kernels per replay outside the V-cycle bodies
  bool batched = false;               // the members' solves run as one batched multigrid loop
};

__global__ void ring_push_kernel(const int* it, const double* meas, int* ring_it, double* ring_meas,
                                 const int* pos) {
  ring_it[*pos] = *it;
  ring_meas[*pos] = *meas;
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

struct Ensemble {
  std::vector<Model*> mem;
  std::vector<cudaStream_t> old_streams, streams;
  std::vector<cudaEvent_t> ev_p;
  cudaStream_t s0 = nullptr;
  cudaEvent_t ev_t = nullptr;
  TendParams* d_params = nullptr;
  TendParams* h_params = nullptr;   // page-locked ring of kRing launches' parameters
  std::vector<cudaEvent_t> ev_ring;
  std::vector<cudaEvent_t> ev_k;   // timing pairs around each stream-mode step's batched launch
  double kernel_ms = 0;            // mean device time of the batched launch (stream-mode steps)
  int* d_work = nullptr;
  int* d_done = nullptr;
  int nwork = 0;
  int ring = 0;
  static constexpr int kRing = 4;
  // captured steps
  bool use_graphs = true;
  std::vector<EnsGraph> graphs;
  std::vector<int*> graph_rings;   // the members' report rings the graphs write
  int* d_pos = nullptr;            // ring index of the step a replay runs
  int* d_slot_it = nullptr;        // per member: the captured solve's report slot
  double* d_slot_meas = nullptr;
  int graph_steps = 0;             // steps of the last run that ran as graph replays
  // fork and join events used only inside captures (an event last recorded in a capture may
  // not be waited on outside it)
  cudaEvent_t ev_cf = nullptr;
  std::vector<cudaEvent_t> ev_cj;
  // the members' multigrid solves batched into one loop (when every member's solver allows)
  MGBatch* mgb = nullptr;
  bool mgb_tried = false;
  cudaStream_t cap = nullptr;   // stream that captures the batched loop's body
  // PAWSIM_ENSEMBLE_PHASES=1 (profiling): event nodes between the phases of a captured step
  // (tendency, the members' pre-solve steps, the solves, the projections); the device times of
  // the last replay are printed at the end of a run
  cudaEvent_t ev_ph[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  void drop_graphs() {
    for (EnsGraph& g : graphs) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      cudaFree(g.d_params);
    }
    graphs.clear();
  }
  ~Ensemble() {
    if (s0) cudaStreamSynchronize(s0);
    for (size_t i = 0; i < mem.size() && i < old_streams.size(); ++i) {
      cudaStreamSynchronize(streams[i]);
      mem[i]->s = old_streams[i];
      if (mem[i]->mg) mem[i]->mg->set_stream(old_streams[i]);
      if (mem[i]->dmg) mem[i]->dmg->set_stream(old_streams[i]);
    }
    drop_graphs();
    delete mgb;
    if (cap) cudaStreamDestroy(cap);
    for (cudaStream_t q : streams) cudaStreamDestroy(q);
    for (cudaEvent_t e : ev_p) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_ring) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_k) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_cj) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_ph)
      if (e) cudaEventDestroy(e);
    if (ev_cf) cudaEventDestroy(ev_cf);
    if (ev_t) cudaEventDestroy(ev_t);
    if (s0) cudaStreamDestroy(s0);
    cudaFree(d_params);
    cudaFree(d_work);
    cudaFree(d_done);
    cudaFree(d_pos);
    cudaFree(d_slot_it);
    cudaFree(d_slot_meas);
    if (h_params) cudaFreeHost(h_params);
  }
};

static int ensemble_create(Model* const* ms, int n, Ensemble** out) {
  if (n < 1) return fail(PAWSIM_GPU_EBADCONFIG, "an ensemble needs at least one member");
  const pawsim_gpu_config& c0 = ms[0]->c;
  for (int i = 0; i < n; ++i) {
    const Model* m = ms[i];
    const pawsim_gpu_config& c = m->c;
    if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "ensemble members must be initialised");
    if (c.Nlay != c0.Nlay || c.mom_scheme != c0.mom_scheme || c.thick_scheme != c0.thick_scheme ||
        c.use_rl != c0.use_rl)
      return fail(PAWSIM_GPU_EUNSUPPORTED, "ensemble members must share Nlay, the schemes and the rigid lid");
    const bool fraction_drag = base_params(ms[i]).drag_bot || base_params(ms[i]).drag_surf;
    if (c.use_tracer || c.use_buoyancy || c.budgets || fraction_drag || m->bud[0] || m->bud[1] || m->bud[2] || m->bud[3] || m->bud[4])
      return fail(PAWSIM_GPU_EUNSUPPORTED, "ensemble members without tracer, budgets or fraction-depth drag");
    for (int j = 0; j < i; ++j)
      if (ms[j] == m) return fail(PAWSIM_GPU_EBADCONFIG, "a model appears twice in the ensemble");
  }
  // every member must take the same kernel instantiation and shared-memory size
  const TendParams p0 = base_params(ms[0]);
  const int ty = tendency_tile_height(p0, c0.thick_scheme);
  for (int i = 1; i < n; ++i) {
    const TendParams pi = base_params(ms[i]);
    if (tendency_tile_height(pi, c0.thick_scheme) != ty || (pi.use_wdia != 0) != (p0.use_wdia != 0) ||
        pi.use_smag != p0.use_smag || (pi.use_fractions != 0) != (p0.use_fractions != 0) ||
        (pi.useA4 != 0) != (p0.useA4 != 0) || (pi.corners != nullptr) != (p0.corners != nullptr) ||
        tendency_lean(pi) != tendency_lean(p0))
      return fail(PAWSIM_GPU_EUNSUPPORTED, "ensemble members must share the tendency kernel's feature set");
  }
  Ensemble* e = new Ensemble();
  e->mem.assign(ms, ms + n);
  std::vector<int> work;
  for (int i = 0; i < n; ++i) {
    const int tiles = ((ms[i]->Nx + 31) / 32) * ((ms[i]->Ny + ty - 1) / ty);
    if (tiles > 0xfffff || i > 2047) {
      delete e;
      return fail(PAWSIM_GPU_EUNSUPPORTED, "ensemble too large for the work-list encoding");
    }
    for (int t = 0; t < tiles; ++t) work.push_back(i << 20 | t);
  }
  e->nwork = (int)work.size();
  bool ok = cudaStreamCreateWithFlags(&e->s0, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->ev_t, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->ev_cf, cudaEventDisableTiming) == cudaSuccess &&
            cudaMalloc(&e->d_params, n * sizeof(TendParams)) == cudaSuccess &&
            cudaMallocHost(&e->h_params, (size_t)Ensemble::kRing * n * sizeof(TendParams)) == cudaSuccess &&
            cudaMalloc(&e->d_work, work.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&e->d_done, sizeof(int)) == cudaSuccess &&
            cudaMemset(e->d_done, 0, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&e->d_pos, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&e->d_slot_it, n * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&e->d_slot_meas, n * sizeof(double)) == cudaSuccess &&
            cudaMemcpy(e->d_work, work.data(), work.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  for (int q = 0; ok && q < Ensemble::kRing; ++q) {
    cudaEvent_t ev;
    ok = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (ok) e->ev_ring.push_back(ev);
  }
  for (int i = 0; ok && i < n; ++i) {
    cudaStream_t q;
    cudaEvent_t ev, evj;
    ok = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&evj, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) break;
    PAWSIM_CUDA_OK(cudaStreamSynchronize(ms[i]->s));
    e->streams.push_back(q);
    e->ev_p.push_back(ev);
    e->ev_cj.push_back(evj);
    e->old_streams.push_back(ms[i]->s);
    ms[i]->s = q;
    if (ms[i]->mg) ms[i]->mg->set_stream(q);
    if (ms[i]->dmg) ms[i]->dmg->set_stream(q);
  }
  if (ok && getenv("PAWSIM_ENSEMBLE_PHASES"))
    for (cudaEvent_t& ev : e->ev_ph) ok = ok && cudaEventCreate(&ev) == cudaSuccess;
  if (!ok) {
    delete e;
    return fail(PAWSIM_GPU_ECUDA, "ensemble set-up failed");
  }
  *out = e;
  return 0;
}

// Can member m's step run as part of a captured graph? (the history shifts, the correction
// needs no host and its multigrid loop is built; SOR's cooperative launch stays on streams)
static bool graph_step_ok(const Model* m, bool shift) {
  if (!shift || !async_correct_ok(m)) return false;
  if (!m->c.use_rl) return true;
  return m->c.solver == PAWSIM_GPU_SOLVER_MG && (m->c.pi_guess != 1 || m->pi_solves >= 2);
}

// The host-side effects of one replayed step of member m: those the captured step's own
// enqueue made (integrator bookkeeping, two corner fills, the correction's flags).
static void replay_member(Model* m, const TendParams& p, bool shift) {
  step_finish(m, p, shift);
  m->thickness_fixed = false;
  if (m->c.use_rl && m->c.solver == PAWSIM_GPU_SOLVER_MG && m->c.pi_guess == 1) ++m->pi_solves;
}

// One member's part of a step on its own stream, after the batched launch (event ev_t): corner
// shadow of the step's start state, bookkeeping, correction with its report to (it, meas).
static int member_step(Ensemble* e, int i, const TendParams& p, bool shift, int* it, double* meas, cudaEvent_t fork) {
  Model* m = e->mem[i];
  PAWSIM_CUDA_OK(cudaStreamWaitEvent(m->s, fork, 0));
  corner_fill(m, m->cur);
  step_finish(m, p, shift);
  return pressure_correct_async(m, it, meas);
}

// The batched multigrid of all members, built once when every member solves with the
// multigrid and its solver allows batching (MGBatch::ok); nullptr otherwise.
static MGBatch* ensemble_mg_batch(Ensemble* e) {
  if (e->mgb_tried) return e->mgb;
  e->mgb_tried = true;
  std::vector<Multigrid*> mgs;
  std::vector<double> tol;
  std::vector<int> maxit;
  std::vector<int*> its;
  std::vector<double*> meas;
  for (size_t i = 0; i < e->mem.size(); ++i) {
    Model* m = e->mem[i];
    if (!m->c.use_rl || m->c.solver != PAWSIM_GPU_SOLVER_MG || !m->mg) return nullptr;
    mgs.push_back(m->mg);
    tol.push_back(m->c.pi_tol);
    maxit.push_back(m->c.maxiters);
    its.push_back(e->d_slot_it + i);
    meas.push_back(e->d_slot_meas + i);
  }
  MGBatch* b = new MGBatch(mgs, tol, maxit, its, meas);
  if (!b->ok()) {
    delete b;
    cudaGetLastError();
    return nullptr;
  }
  e->mgb = b;
  return b;
}

// Capture one step of every member into graph g (its parameter blocks already in g.d_params).
// With the batched multigrid: each member's pre-solve steps on its stream, the one batched
// loop on the launch stream, then each member's projection.
static int ensemble_capture(Ensemble* e, EnsGraph& g, const std::vector<TendParams>& p,
                            const std::vector<char>& shift) {
  const int n = (int)e->mem.size();
  MGBatch* mgb = ensemble_mg_batch(e);
  const long long g0 = g_launches;
  PAWSIM_CUDA_OK(cudaStreamBeginCapture(e->s0, cudaStreamCaptureModeRelaxed));
  int rc = 0;
  auto phase = [&](int k) {
    if (e->ev_ph[k]) cudaEventRecordWithFlags(e->ev_ph[k], e->s0, cudaEventRecordExternal);
  };
  phase(0);
  const int nl = launch_tendency_batch(p[0], g.d_params, e->d_work, e->nwork, n, e->d_done,
                                       e->mem[0]->c.mom_scheme, e->mem[0]->c.thick_scheme, e->s0);
  if (nl < 0) rc = fail(PAWSIM_GPU_EUNSUPPORTED, "batched tendency launch not available");
  g_launches += nl > 0 ? nl : 0;
  phase(1);
  if (!rc && cudaEventRecord(e->ev_cf, e->s0) != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "event record failed");
  if (mgb) {
    g.batched = true;
    for (int i = 0; i < n && !rc; ++i) {
      Model* m = e->mem[i];
      if (cudaStreamWaitEvent(m->s, e->ev_cf, 0) != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "capture fork failed");
      if (rc) break;
      corner_fill(m, m->cur);
      step_finish(m, p[i], shift[i] != 0);
      rc = pressure_pre_solve(m);
      if (!rc && (cudaEventRecord(e->ev_cj[i], m->s) != cudaSuccess ||
                  cudaStreamWaitEvent(e->s0, e->ev_cj[i], 0) != cudaSuccess))
        rc = fail(PAWSIM_GPU_ECUDA, "capture join failed");
    }
    phase(2);
    if (!rc && mgb->capture(e->s0, e->cap) != 0) rc = fail(PAWSIM_GPU_ECUDA, "batched multigrid capture failed");
    phase(3);
    if (!rc && cudaEventRecord(e->ev_cf, e->s0) != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "event record failed");
    for (int i = 0; i < n && !rc; ++i) {
      Model* m = e->mem[i];
      if (cudaStreamWaitEvent(m->s, e->ev_cf, 0) != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "capture fork failed");
      if (rc) break;
      rc = pressure_post_solve(m);
      if (rc) break;
      ring_push_kernel<<<1, 1, 0, m->s>>>(e->d_slot_it + i, e->d_slot_meas + i, m->run_iters, m->run_meas, e->d_pos);
      ++g_launches;
      if (cudaEventRecord(e->ev_cj[i], m->s) != cudaSuccess || cudaStreamWaitEvent(e->s0, e->ev_cj[i], 0) != cudaSuccess)
        rc = fail(PAWSIM_GPU_ECUDA, "capture join failed");
    }
  }
  for (int i = 0; i < n && !rc && !mgb; ++i) {
    Model* m = e->mem[i];
    rc = member_step(e, i, p[i], shift[i] != 0, e->d_slot_it + i, e->d_slot_meas + i, e->ev_cf);
    if (rc) break;
    ring_push_kernel<<<1, 1, 0, m->s>>>(e->d_slot_it + i, e->d_slot_meas + i, m->run_iters, m->run_meas, e->d_pos);
    ++g_launches;
    if (cudaEventRecord(e->ev_cj[i], m->s) != cudaSuccess || cudaStreamWaitEvent(e->s0, e->ev_cj[i], 0) != cudaSuccess)
      rc = fail(PAWSIM_GPU_ECUDA, "capture join failed");
  }
  phase(4);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(e->s0, &graph);
  if (!rc && ce != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "ensemble step capture failed");
  if (!rc && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) rc = fail(PAWSIM_GPU_ECUDA, "ensemble graph instantiation failed");
  if (graph) cudaGraphDestroy(graph);
  g.launches = g_launches - g0;
  return rc;
}

static int ensemble_run(Ensemble* e, unsigned n0, unsigned nsteps) {
  const int n = (int)e->mem.size();
  // the rings keep their size across runs so that captured graphs stay valid
  std::vector<int*> rings(n);
  for (int i = 0; i < n; ++i) {
    Model* m = e->mem[i];
    m->last_run_iters.assign(nsteps, 0);
    if (!ensure_run_ring(m, nsteps > 1024u ? nsteps : 1024u)) return fail(PAWSIM_GPU_ECUDA, "run report allocation failed");
    rings[i] = m->run_iters;
  }
  if (rings != e->graph_rings) {
    PAWSIM_CUDA_OK(cudaStreamSynchronize(e->s0));
    e->drop_graphs();
    e->graph_rings = rings;
  }
  while (e->ev_k.size() < 2 * (size_t)nsteps) {
    cudaEvent_t ev;
    PAWSIM_CUDA_OK(cudaEventCreate(&ev));
    e->ev_k.push_back(ev);
  }
  std::vector<std::vector<char>> async(n, std::vector<char>(nsteps, 0));
  std::vector<char> timed(nsteps, 0), batched(nsteps, 0);
  std::vector<TendParams> p(n);
  std::vector<char> shift(n);
  std::vector<int> key(5 * n);
  e->graph_steps = 0;
  for (unsigned q = 0; q < nsteps; ++q) {
    const unsigned step = n0 + q;
    bool graph_ok = e->use_graphs;
    for (int i = 0; i < n; ++i) {
      Model* m = e->mem[i];
      bool sh = true;
      p[i] = step_params(m, step, true, &sh);
      shift[i] = sh;
      graph_ok = graph_ok && graph_step_ok(m, sh);
      key[5 * i] = m->cur; key[5 * i + 1] = m->h1; key[5 * i + 2] = m->h2; key[5 * i + 3] = m->h3;
      key[5 * i + 4] = m->corner_cur;
    }
    // every step waits for the members' last corrections (events of stream-mode steps; after a
    // replay the launch stream is already ordered behind them)
    for (int i = 0; i < n; ++i) PAWSIM_CUDA_OK(cudaStreamWaitEvent(e->s0, e->ev_p[i], 0));
    const int r = e->ring;
    e->ring = (e->ring + 1) % Ensemble::kRing;
    PAWSIM_CUDA_OK(cudaEventSynchronize(e->ev_ring[r]));   // that slot's earlier copy is done
    TendParams* hp = e->h_params + (size_t)r * n;
    for (int i = 0; i < n; ++i) hp[i] = p[i];
    if (graph_ok) {
      EnsGraph* g = nullptr;
      for (EnsGraph& c : e->graphs)
        if (c.key == key) g = &c;
      const bool fresh = g == nullptr;
      if (fresh) {
        if (e->graphs.size() >= 12) {
          PAWSIM_CUDA_OK(cudaStreamSynchronize(e->s0));
          e->drop_graphs();
        }
        e->graphs.emplace_back();
        g = &e->graphs.back();
        g->key = key;
        PAWSIM_CUDA_OK(cudaMalloc(&g->d_params, n * sizeof(TendParams)));
      }
      if (fresh || memcmp(g->h_params.data(), p.data(), n * sizeof(TendParams)) != 0) {
        // the blocks change only with time-dependent forcing records
        PAWSIM_CUDA_OK(cudaMemcpyAsync(g->d_params, hp, n * sizeof(TendParams), cudaMemcpyHostToDevice, e->s0));
        g->h_params = p;
      }
      PAWSIM_CUDA_OK(cudaEventRecord(e->ev_ring[r], e->s0));
      set_int_kernel<<<1, 1, 0, e->s0>>>(e->d_pos, (int)q);
      ++g_launches;
      if (fresh) {
        const int rc = ensemble_capture(e, *g, p, shift);
        if (rc) {
          PAWSIM_CUDA_OK(cudaStreamSynchronize(e->s0));
          e->drop_graphs();
          return rc;
        }
      } else {
        g_launches += g->launches;
        for (int i = 0; i < n; ++i) replay_member(e->mem[i], p[i], shift[i] != 0);
      }
      PAWSIM_CUDA_OK(cudaGraphLaunch(g->exec, e->s0));
      for (int i = 0; i < n; ++i) async[i][q] = 1;
      batched[q] = g->batched ? 1 : 0;
      ++e->graph_steps;
      continue;
    }
    // stream mode. Phase 1: the fused kernels of all members in one launch
    PAWSIM_CUDA_OK(cudaMemcpyAsync(e->d_params, hp, n * sizeof(TendParams), cudaMemcpyHostToDevice, e->s0));
    PAWSIM_CUDA_OK(cudaEventRecord(e->ev_ring[r], e->s0));
    PAWSIM_CUDA_OK(cudaEventRecord(e->ev_k[2 * q], e->s0));
    const int nl = launch_tendency_batch(p[0], e->d_params, e->d_work, e->nwork, n, e->d_done,
                                         e->mem[0]->c.mom_scheme, e->mem[0]->c.thick_scheme, e->s0);
    if (nl < 0) return fail(PAWSIM_GPU_EUNSUPPORTED, "batched tendency launch not available");
    g_launches += nl;
    PAWSIM_CUDA_OK(cudaEventRecord(e->ev_k[2 * q + 1], e->s0));
    timed[q] = 1;
    PAWSIM_CUDA_OK(cudaEventRecord(e->ev_t, e->s0));
    // phase 2: each member's corner shadow, bookkeeping and correction on its own stream
    for (int i = 0; i < n; ++i) {
      Model* m = e->mem[i];
      if (async_correct_ok(m)) {
        int rc = member_step(e, i, p[i], shift[i] != 0, m->run_iters + q, m->run_meas + q, e->ev_t);
        if (rc) return rc;
        async[i][q] = 1;
      } else {
        PAWSIM_CUDA_OK(cudaStreamWaitEvent(m->s, e->ev_t, 0));
        corner_fill(m, m->cur);
        step_finish(m, p[i], shift[i] != 0);
        pawsim_gpu_stats st;
        const int it = pressure_correct(m, 1, &st);
        if (it < 0) return it;
        m->last_run_iters[q] = it;
      }
      PAWSIM_CUDA_OK(cudaEventRecord(e->ev_p[i], m->s));
    }
  }
  // the reports of the run, read once; the failure options as pawsim_gpu_run applies them
  PAWSIM_CUDA_OK(cudaStreamSynchronize(e->s0));
  int r = 0;
  std::vector<int> most(nsteps, 0);   // cycles of a batched loop: those of its slowest member
  for (int i = 0; i < n; ++i) {
    Model* m = e->mem[i];
    std::vector<int> it(nsteps);
    PAWSIM_CUDA_OK(cudaMemcpyAsync(it.data(), m->run_iters, nsteps * sizeof(int), cudaMemcpyDeviceToHost, m->s));
    PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
    for (unsigned q = 0; q < nsteps; ++q) {
      if (!async[i][q]) continue;
      m->last_run_iters[q] = it[q];
      if (batched[q]) most[q] = std::max(most[q], it[q]);
      else if (m->c.use_rl && m->c.solver == PAWSIM_GPU_SOLVER_MG) g_launches += (long long)it[q] * m->mg->body_launches();
    }
    for (unsigned q = 0; q < nsteps && !r; ++q) r = check_converged(m, m->last_run_iters[q]);
    if (!r && m->nonfinite) {
      m->nf_calls = m->c.check_nonfinite - 1;
      r = check_state_finite(m);
    }
  }
  for (unsigned q = 0; q < nsteps; ++q)
    if (batched[q] && e->mgb) g_launches += (long long)most[q] * e->mgb->body_launches();
  double tot = 0;
  int cnt = 0;
  for (unsigned q = 0; q < nsteps; ++q) {
    if (!timed[q]) continue;
    float ms = 0;
    PAWSIM_CUDA_OK(cudaEventElapsedTime(&ms, e->ev_k[2 * q], e->ev_k[2 * q + 1]));
    tot += ms;
    ++cnt;
  }
  e->kernel_ms = cnt ? tot / cnt : 0;
  if (e->ev_ph[0] && e->graph_steps) {
    float t[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&t[k], e->ev_ph[k], e->ev_ph[k + 1]);
    fprintf(stderr, "pawsim ensemble phases (ms, last replay): tendency %.3f pre-solve %.3f solves %.3f post %.3f\n",
            t[0], t[1], t[2], t[3]);
  }
  return r;
}

}  // namespace pawsim

using namespace pawsim;

struct pawsim_gpu {
  Model* m;
};

extern "C" {

int pawsim_gpu_create(const pawsim_gpu_config* cfg, pawsim_gpu** out) {
  if (!cfg || !out) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  Model* m = nullptr;
  int r = create(cfg, &m);
  if (r) return r;
  *out = new pawsim_gpu{m};
  return 0;
}

void pawsim_gpu_destroy(pawsim_gpu* h) {
  if (!h) return;
  delete h->m;
  delete h;
}

int pawsim_gpu_set_field(pawsim_gpu* h, const char* name, int k, const double* host, size_t n) {
  if (!h || !host) return fail(PAWSIM_GPU_EBADNAME, "null argument");
  return set_field(h->m, name, k, host, n);
}

int pawsim_gpu_get_field(pawsim_gpu* h, const char* name, int k, double* host, size_t n) {
  if (!h || !host) return fail(PAWSIM_GPU_EBADNAME, "null argument");
  return get_field(h->m, name, k, host, n);
}

int pawsim_gpu_init(pawsim_gpu* h) { return h ? init(h->m) : PAWSIM_GPU_EBADCONFIG; }

int pawsim_gpu_tendency_eval(pawsim_gpu* h) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  int r = tendency_eval(h->m);
  if (r) return r;
  PAWSIM_CUDA_OK(cudaStreamSynchronize(h->m->s));
  return 0;
}

int pawsim_gpu_integrator_step(pawsim_gpu* h, unsigned n) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  int r = integrator_step(h->m, n, false);
  if (r) return r;
  return check_state_finite(h->m);
}

int pawsim_gpu_pressure_correct(pawsim_gpu* h, int update_diags, pawsim_gpu_stats* st) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  int r = pressure_correct(h->m, update_diags, st);
  if (r < 0) return r;
  return check_converged(h->m, r);
}

int pawsim_gpu_prelim(pawsim_gpu* h, pawsim_gpu_stats* st) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (!m->ready) {
    int r = init(m);
    if (r) return r;
  }
  m->thickness_fixed = false;
  int r = pressure_correct(m, 0, st);
  if (r < 0) return r;
  r = tendency_eval(m);   // rebuilds wdia for the n = 0 output, as pawsim.c:296-300 does
  if (r) return r;
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  return 0;
}

int pawsim_gpu_step(pawsim_gpu* h, unsigned n, pawsim_gpu_stats* st) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  int r = integrator_step(h->m, n, true);
  if (r) return r;
  const int iters = pressure_correct(h->m, 1, st);
  if (iters < 0) return iters;
  r = check_state_finite(h->m);
  if (r) return r;
  return check_converged(h->m, iters);
}

int pawsim_gpu_run(pawsim_gpu* h, unsigned n0, unsigned nsteps, pawsim_gpu_stats* st) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  m->last_run_iters.assign(nsteps, 0);
  if (nsteps == 0) return 0;
  if (!ensure_run_ring(m, nsteps)) return fail(PAWSIM_GPU_ECUDA, "run report allocation failed");
  // steps whose correction needs the host run synchronously (the first solves tune the
  // multigrid and build its graph); the others are enqueued back to back and their reports
  // read once at the end
  std::vector<char> async(nsteps, 0);
  pawsim_gpu_stats last;
  memset(&last, 0, sizeof(last));
  for (unsigned q = 0; q < nsteps; ++q) {
    const unsigned n = n0 + q;
    if (async_correct_ok(m)) {
      int r = integrator_step(m, n, true);
      if (r) return r;
      r = pressure_correct_async(m, m->run_iters + q, m->run_meas + q);
      if (r) return r;
      async[q] = 1;
    } else {
      int r = pawsim_gpu_step(h, n, &last);
      if (r) return r;
      m->last_run_iters[q] = last.iters;
    }
  }
  std::vector<int> it(nsteps);
  std::vector<double> ms(nsteps);
  PAWSIM_CUDA_OK(cudaMemcpyAsync(it.data(), m->run_iters, nsteps * sizeof(int), cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaMemcpyAsync(ms.data(), m->run_meas, nsteps * sizeof(double), cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  int r = 0;
  for (unsigned q = 0; q < nsteps; ++q) {
    if (!async[q]) continue;
    m->last_run_iters[q] = it[q];
    if (m->c.use_rl && m->c.solver == PAWSIM_GPU_SOLVER_MG) g_launches += (long long)it[q] * m->mg->body_launches();
    if (!r) r = check_converged(m, it[q]);
    if (q == nsteps - 1) {
      last.iters = it[q];
      last.stop_measure = m->c.solver == PAWSIM_GPU_SOLVER_MG ? ms[q] : 0;
      last.mg_omega = m->mg && m->c.solver == PAWSIM_GPU_SOLVER_MG ? m->mg->omega() : 0;
    }
  }
  if (st) *st = last;
  if (m->nonfinite) {   // the flag raised during the run, read once
    m->nf_calls = m->c.check_nonfinite - 1;
    int rf = check_state_finite(m);
    if (rf) return rf;
  }
  return r;
}

struct pawsim_gpu_ensemble {
  Ensemble* e;
};

int pawsim_gpu_ensemble_create(pawsim_gpu* const* members, int n, pawsim_gpu_ensemble** out) {
  if (!members || !out || n < 1) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  std::vector<Model*> ms(n);
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return fail(PAWSIM_GPU_EBADCONFIG, "null member");
    ms[i] = members[i]->m;
  }
  Ensemble* e = nullptr;
  int r = ensemble_create(ms.data(), n, &e);
  if (r) return r;
  *out = new pawsim_gpu_ensemble{e};
  return 0;
}

int pawsim_gpu_ensemble_run(pawsim_gpu_ensemble* h, unsigned n0, unsigned nsteps) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  return ensemble_run(h->e, n0, nsteps);
}

double pawsim_gpu_ensemble_kernel_ms(const pawsim_gpu_ensemble* h) {
  return h ? h->e->kernel_ms : 0;
}

int pawsim_gpu_ensemble_set_graphs(pawsim_gpu_ensemble* h, int on) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  h->e->use_graphs = on != 0;
  return 0;
}

int pawsim_gpu_ensemble_graph_steps(const pawsim_gpu_ensemble* h) {
  return h ? h->e->graph_steps : 0;
}

int pawsim_gpu_ensemble_batched_mg(const pawsim_gpu_ensemble* h) {
  return h && h->e->mgb ? 1 : 0;
}

void pawsim_gpu_ensemble_destroy(pawsim_gpu_ensemble* h) {
  if (!h) return;
  delete h->e;
  delete h;
}

int pawsim_gpu_run_iterations(pawsim_gpu* h, int* iters, size_t n) {
  if (!h || !iters) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  const std::vector<int>& v = h->m->last_run_iters;
  if (n != v.size()) return fail(PAWSIM_GPU_EBADCONFIG, "n must equal the last run's step count");
  if (n) memcpy(iters, v.data(), n * sizeof(int));
  return 0;
}

int pawsim_gpu_accumulate_averages(pawsim_gpu* h, double avg_fac) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  if (!m->avg) {
    m->avg = m->alloc<double>(avg_elems(m));
    if (!m->avg) return fail(PAWSIM_GPU_ECUDA, "average storage allocation failed");
  }
  const size_t ls = m->lstride;
  double* b = m->avg;
  AvgParams a;
  a.dtfac = avg_fac * m->c.dt;   // dtfac of diagnostics.c:337
  a.use_rl = m->c.use_rl;
  a.h0 = m->c.h0;
  for (int k = 0; k < m->L; ++k) { a.gg[k] = m->gg[k]; a.geff[k] = m->geff[k]; }
  a.u = m->u[m->cur]; a.v = m->v[m->cur]; a.h = m->h[m->cur];
  a.pi = m->pi; a.hhb = m->hhb; a.wdia = m->wdia;
  const size_t Ls = (size_t)m->L * ls;
  a.au = b; a.av = b + Ls; a.ah = b + 2 * Ls; a.aM = b + 3 * Ls; a.ahu = b + 4 * Ls; a.ahv = b + 5 * Ls;
  a.ahuu = b + 6 * Ls; a.ahvv = b + 7 * Ls; a.ahuv = b + 8 * Ls; a.aW = b + 9 * Ls; a.api = a.aW + Ls + ls;
  a.b = m->b[0] ? m->b[m->cur] : nullptr;
  a.use_buoy = m->c.use_buoyancy;
  a.ab = m->b[0] ? a.api + ls : nullptr;
  corner_fill(m, m->cur);   // the averages reload the state (diagnostics.c:320-324)
  launch_accumulate_averages(m->grid2(), a, m->s);
  ++g_launches;
  PAWSIM_CUDA_OK(cudaGetLastError());
  return 0;
}

int pawsim_gpu_scale_averages(pawsim_gpu* h, double factor) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (!m->avg) return fail(PAWSIM_GPU_EBADCONFIG, "no averages accumulated");
  launch_scale(m->avg, avg_elems(m), factor, m->s);
  ++g_launches;
  PAWSIM_CUDA_OK(cudaGetLastError());
  return 0;
}

int pawsim_gpu_zero_averages(pawsim_gpu* h) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (m->avg)
    PAWSIM_CUDA_OK(cudaMemsetAsync(m->avg, 0, avg_elems(m) * sizeof(double), m->s));
  return 0;
}

int pawsim_gpu_scale_budgets(pawsim_gpu* h, int mask, double factor) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  for (int f = 0; f < 5; ++f)
    if ((mask & (1 << f)) && m->bud[f]) {
      launch_scale(m->bud[f], (size_t)kBudgetTerms[f] * m->L * m->lstride, factor, m->s);
      ++g_launches;
    }
  PAWSIM_CUDA_OK(cudaGetLastError());
  return 0;
}

int pawsim_gpu_zero_budgets(pawsim_gpu* h, int mask) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  for (int f = 0; f < 5; ++f)
    if ((mask & (1 << f)) && m->bud[f])
      PAWSIM_CUDA_OK(cudaMemsetAsync(m->bud[f], 0, (size_t)kBudgetTerms[f] * m->L * m->lstride * sizeof(double), m->s));
  return 0;
}

int pawsim_gpu_energy(pawsim_gpu* h, int eta_from_step_start, double* KE, double* PE, double* Z) {
  if (!h || !KE || !PE || !Z) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  Model* m = h->m;
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  if (eta_from_step_start && !m->prev_h)
    return fail(PAWSIM_GPU_EBADCONFIG, "no step since the thickness was loaded");
  const Grid2 g = m->grid2();
  const bool serial = m->serial();
  const size_t need = ez_scratch_elems(g, serial);
  if (m->ez_elems < need) {
    double* p = m->alloc<double>(need);
    if (!p) return fail(PAWSIM_GPU_ECUDA, "energy scratch allocation failed");
    m->ez = p;   // an earlier, smaller buffer stays in the model's list until it is destroyed
    m->ez_elems = need;
  }
  if (!m->ez_out) {
    m->ez_out = m->alloc<double>(AVG_LMAX + 2);
    if (!m->ez_out) return fail(PAWSIM_GPU_ECUDA, "energy scratch allocation failed");
  }
  EzParams e;
  e.h0 = m->c.h0;
  for (int k = 0; k < m->L; ++k) e.geff[k] = m->geff[k];
  e.u = m->u[m->cur]; e.v = m->v[m->cur]; e.h = m->h[m->cur];
  e.hw = eta_from_step_start ? m->h[1 - m->cur] : m->h[m->cur];
  e.hhb = m->hhb; e.omz = m->omz; e.qpitch = m->qpitch;
  e.b = m->c.use_buoyancy ? m->b[m->cur] : nullptr;
  g_launches += launch_energy(g, e, serial, m->ez, m->ez_out, m->s);
  PAWSIM_CUDA_OK(cudaGetLastError());
  double out[AVG_LMAX + 2];
  PAWSIM_CUDA_OK(cudaMemcpyAsync(out, m->ez_out, (m->L + 2) * sizeof(double), cudaMemcpyDeviceToHost, m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  *KE = out[0];
  *PE = out[1];
  for (int k = 0; k < m->L; ++k) Z[k] = out[2 + k];
  return 0;
}

// planes of one save, in file order: u, v, h (and b) per layer, w_dia per interface, pi
static size_t save_plane_count(const Model* m) {
  return (size_t)m->L * (m->c.use_tracer ? 4 : 3) + (m->L + 1) + (m->c.use_rl ? 1 : 0);
}

int pawsim_gpu_save_begin(pawsim_gpu* h, int* slot_out) {
  if (!h || !slot_out) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  Model* m = h->m;
  if (!m->ready) return fail(PAWSIM_GPU_EBADCONFIG, "pawsim_gpu_init must follow the uploads");
  const size_t N = (size_t)m->Nx * m->Ny;
  if (!m->copy_s) {
    PAWSIM_CUDA_OK(cudaGetDevice(&m->device));
    PAWSIM_CUDA_OK(cudaStreamCreateWithFlags(&m->copy_s, cudaStreamNonBlocking));
    m->save_planes = save_plane_count(m);
    for (Model::SaveSlot& q : m->save) {
      q.dev = m->alloc<double>(m->save_planes * N);
      if (!q.dev) return fail(PAWSIM_GPU_ECUDA, "save staging allocation failed");
      PAWSIM_CUDA_OK(cudaMallocHost(&q.host, m->save_planes * N * sizeof(double)));
      PAWSIM_CUDA_OK(cudaEventCreateWithFlags(&q.staged, cudaEventDisableTiming));
      PAWSIM_CUDA_OK(cudaEventCreateWithFlags(&q.done, cudaEventDisableTiming));
    }
  }
  const int sl = m->save_next;
  Model::SaveSlot& q = m->save[sl];
  {
    // a slot is reused only after its previous contents were handed back
    std::unique_lock<std::mutex> lk(m->save_mu);
    if (!m->save_cv.wait_for(lk, std::chrono::seconds(600), [&] { return !q.busy; }))
      return fail(PAWSIM_GPU_EBADCONFIG, "no save slot was released within 600 s");
    q.busy = true;
  }
  m->save_next ^= 1;
  std::vector<const double*> src;
  const int cur = m->cur;
  for (int k = 0; k < m->L; ++k) {
    src.push_back(m->u[cur] + k * m->lstride);
    src.push_back(m->v[cur] + k * m->lstride);
    src.push_back(m->h[cur] + k * m->lstride);
    if (m->c.use_tracer) src.push_back(m->b[cur] + k * m->lstride);
  }
  for (int k = 0; k <= m->L; ++k) src.push_back(m->wdia + k * m->lstride);
  if (m->c.use_rl) src.push_back(m->pi);
  // the slot's previous copy-out (if any) must be finished before the slot is refilled;
  // pack on the model's stream (ordered with the steps), then copy out on the copy stream
  PAWSIM_CUDA_OK(cudaStreamWaitEvent(m->s, q.done, 0));
  for (size_t p = 0; p < src.size(); ++p)
    PAWSIM_CUDA_OK(cudaMemcpy2DAsync(q.dev + p * N, m->Nx * sizeof(double), src[p], m->pitch * sizeof(double),
                                     m->Nx * sizeof(double), m->Ny, cudaMemcpyDeviceToDevice, m->s));
  PAWSIM_CUDA_OK(cudaEventRecord(q.staged, m->s));
  PAWSIM_CUDA_OK(cudaStreamWaitEvent(m->copy_s, q.staged, 0));
  PAWSIM_CUDA_OK(cudaMemcpyAsync(q.host, q.dev, src.size() * N * sizeof(double), cudaMemcpyDeviceToHost, m->copy_s));
  PAWSIM_CUDA_OK(cudaEventRecord(q.done, m->copy_s));
  *slot_out = sl;
  return 0;
}

int pawsim_gpu_save_wait(pawsim_gpu* h, int slot, const double** host) {
  if (!h || !host || slot < 0 || slot > 1) return fail(PAWSIM_GPU_EBADCONFIG, "bad argument");
  Model* m = h->m;
  Model::SaveSlot& q = m->save[slot];
  {
    std::lock_guard<std::mutex> lk(m->save_mu);
    if (!q.busy) return fail(PAWSIM_GPU_EBADCONFIG, "slot holds no save");
  }
  PAWSIM_CUDA_OK(cudaSetDevice(m->device));
  PAWSIM_CUDA_OK(cudaEventSynchronize(q.done));
  *host = q.host;
  return 0;
}

int pawsim_gpu_save_release(pawsim_gpu* h, int slot) {
  if (!h || slot < 0 || slot > 1) return fail(PAWSIM_GPU_EBADCONFIG, "bad argument");
  Model* m = h->m;
  {
    std::lock_guard<std::mutex> lk(m->save_mu);
    m->save[slot].busy = false;
  }
  m->save_cv.notify_all();
  return 0;
}

size_t pawsim_gpu_save_planes(const pawsim_gpu* h) { return h ? save_plane_count(h->m) : 0; }

int pawsim_gpu_solve_mg(pawsim_gpu* h, pawsim_gpu_stats* st) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (!m->mg) return fail(PAWSIM_GPU_EBADCONFIG, "multigrid not configured");
  double mres = 0;
  PAWSIM_CUDA_OK(cudaEventRecord(m->ev0, m->s));
  int it = m->mg->solve(m->pi, m->pitch, m->rhs, m->pitch, m->c.pi_tol, m->c.maxiters, &mres);
  if (it < 0) return fail(PAWSIM_GPU_ECUDA, "multigrid solve failed (graph build or stream error)");
  PAWSIM_CUDA_OK(cudaEventRecord(m->ev1, m->s));
  PAWSIM_CUDA_OK(cudaStreamSynchronize(m->s));
  if (st) {
    memset(st, 0, sizeof(*st));
    st->iters = it;
    st->stop_measure = mres;
    st->mg_omega = m->mg->omega();
    float ms = 0;
    cudaEventElapsedTime(&ms, m->ev0, m->ev1);
    st->solve_ms = ms;
  }
  return 0;
}

int pawsim_gpu_set_stream(pawsim_gpu* h, void* stream) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  h->m->s = (cudaStream_t)stream;
  if (h->m->mg) h->m->mg->set_stream(h->m->s);
  if (h->m->dmg) h->m->dmg->set_stream(h->m->s);
  return 0;
}

int pawsim_gpu_synchronize(pawsim_gpu* h) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  PAWSIM_CUDA_OK(cudaStreamSynchronize(h->m->s));
  return 0;
}

double pawsim_gpu_time(const pawsim_gpu* h) { return h ? h->m->t : 0.0; }

long long pawsim_gpu_launch_count(const pawsim_gpu* h) {
  (void)h;
  return g_launches;
}

const char* pawsim_gpu_last_error(void) { return g_err; }

int pawsim_gpu_nn_setup(pawsim_gpu* h, int mode, int max_pairs, int batch, unsigned long long seed) {
  if (!h) return PAWSIM_GPU_EBADCONFIG;
  Model* m = h->m;
  if (mode && (m->c.solver != PAWSIM_GPU_SOLVER_MG || !m->mg))
    return fail(PAWSIM_GPU_EUNSUPPORTED, "the learned warm start needs the multigrid solver (after init)");
  if (mode && !m->ws) {
    if (!WarmStart::factor(m->Nx, m->Ny))
      return fail(PAWSIM_GPU_EUNSUPPORTED, "grid not supported by the warm-start network");
    if (max_pairs < 1 || batch < 1) return fail(PAWSIM_GPU_EBADCONFIG, "max_pairs and batch must be positive");
    m->ws = new WarmStart(m->Nx, m->Ny, m->pitch, max_pairs, batch, seed, m->s);
    if (!m->ws->ok()) {
      delete m->ws;
      m->ws = nullptr;
      return fail(PAWSIM_GPU_ECUDA, "warm-start allocation failed");
    }
  }
  m->nn_mode = mode;
  return 0;
}

int pawsim_gpu_nn_train(pawsim_gpu* h, int epochs, float lr, double* loss) {
  if (!h || !h->m->ws) return fail(PAWSIM_GPU_EBADCONFIG, "warm start not configured");
  int r = h->m->ws->train(epochs, lr, 1234567ull, loss, h->m->s);
  if (r == -3) return fail(PAWSIM_GPU_ECUDA, "a tensor-core kernel gave up waiting");
  if (r) return fail(PAWSIM_GPU_ECUDA, "warm-start training failed (no pairs, or a CUDA error)");
  return 0;
}

int pawsim_gpu_nn_pairs(pawsim_gpu* h) { return (h && h->m->ws) ? h->m->ws->pairs() : 0; }

void* pawsim_gpu_nn_net(pawsim_gpu* h) { return (h && h->m->ws) ? (void*)h->m->ws->net() : nullptr; }

int pawsim_nn_net_create(int H, int W, int Bmax, unsigned long long seed, void** net) {
  if (!net) return PAWSIM_GPU_EBADCONFIG;
  WarmNet* n = new WarmNet(H, W, Bmax, seed);
  if (!n->ok()) {
    delete n;
    return fail(PAWSIM_GPU_EBADCONFIG, "network sizes must be multiples of 8 (or allocation failed)");
  }
  *net = n;
  return 0;
}

void pawsim_nn_net_destroy(void* net) { delete static_cast<WarmNet*>(net); }

long long pawsim_nn_net_param_count(void* net) {
  return net ? (long long)static_cast<WarmNet*>(net)->param_count() : 0;
}

int pawsim_nn_net_get_params(void* net, float* host, size_t n) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w || !host || n != w->param_count()) return PAWSIM_GPU_EBADCONFIG;
  return w->get_params(host) ? fail(PAWSIM_GPU_ECUDA, "copy failed") : 0;
}

int pawsim_nn_net_set_params(void* net, const float* host, size_t n) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w || !host || n != w->param_count()) return PAWSIM_GPU_EBADCONFIG;
  return w->set_params(host) ? fail(PAWSIM_GPU_ECUDA, "copy failed") : 0;
}

int pawsim_nn_net_get_grads(void* net, float* host, size_t n) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w || !host || n != w->param_count()) return PAWSIM_GPU_EBADCONFIG;
  return w->get_grads(host) ? fail(PAWSIM_GPU_ECUDA, "copy failed") : 0;
}

int pawsim_nn_net_forward(void* net, const void* in, int B, float* out_host) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w || !in || !out_host || B < 1 || B > w->Bmax()) return PAWSIM_GPU_EBADCONFIG;
  if (w->forward(static_cast<const __nv_bfloat16*>(in), B, 0)) return fail(PAWSIM_GPU_ECUDA, "forward failed");
  PAWSIM_CUDA_OK(cudaMemcpy2D(out_host, sizeof(float), w->out(), 16 * sizeof(float), sizeof(float),
                              (size_t)B * w->H() * w->W(), cudaMemcpyDeviceToHost));
  int e = 0;
  PAWSIM_CUDA_OK(cudaMemcpy(&e, w->err(), sizeof(int), cudaMemcpyDeviceToHost));
  return e ? fail(PAWSIM_GPU_ECUDA, "a tensor-core kernel gave up waiting") : 0;
}

int pawsim_nn_net_backward(void* net, const void* in, const float* target, int B, double* loss) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w || !in || !target || B < 1 || B > w->Bmax()) return PAWSIM_GPU_EBADCONFIG;
  double* dl = nullptr;
  PAWSIM_CUDA_OK(cudaMalloc(&dl, sizeof(double)));
  int r = w->backward(static_cast<const __nv_bfloat16*>(in), target, B, dl, 0);
  double hl = 0;
  cudaMemcpy(&hl, dl, sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dl);
  if (r) return fail(PAWSIM_GPU_ECUDA, "backward failed");
  if (loss) *loss = hl;
  int e = 0;
  PAWSIM_CUDA_OK(cudaMemcpy(&e, w->err(), sizeof(int), cudaMemcpyDeviceToHost));
  return e ? fail(PAWSIM_GPU_ECUDA, "a tensor-core kernel gave up waiting") : 0;
}

int pawsim_nn_net_adam(void* net, float lr) {
  WarmNet* w = static_cast<WarmNet*>(net);
  if (!w) return PAWSIM_GPU_EBADCONFIG;
  if (w->adam_step(lr, 0)) return fail(PAWSIM_GPU_ECUDA, "adam step failed");
  PAWSIM_CUDA_OK(cudaDeviceSynchronize());
  return 0;
}

int pawsim_gpu_check_division(const double* x_host, size_t n, double d, long long* bad) {
  if (!x_host || !bad || n == 0) return fail(PAWSIM_GPU_EBADCONFIG, "null argument");
  double* x = nullptr;
  unsigned long long* cnt = nullptr;
  PAWSIM_CUDA_OK(cudaMalloc(&x, n * sizeof(double)));
  PAWSIM_CUDA_OK(cudaMalloc(&cnt, sizeof(unsigned long long)));
  PAWSIM_CUDA_OK(cudaMemcpy(x, x_host, n * sizeof(double), cudaMemcpyHostToDevice));
  PAWSIM_CUDA_OK(cudaMemset(cnt, 0, sizeof(unsigned long long)));
  div_check_kernel<<<(unsigned)((n + 255) / 256), 256>>>(x, n, d, 1.0 / d, cnt);
  ++g_launches;
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpy(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(x);
  cudaFree(cnt);
  if (e != cudaSuccess) return set_cuda_error(e, "check_division", __FILE__, __LINE__);
  *bad = (long long)h;
  return 0;
}

}  // extern "C"
