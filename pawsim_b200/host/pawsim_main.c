/*
 * pawsim_main.c -- drop-in host driver: PAWSIM_B200.exe <input_file> <output_dir>
 *
 * Same command line, parameter file, input data files, output files and stdout lines as
 * the reference's serial executable (model_code/pawsim.c:363-525), with the hot path on
 * the GPU through the C ABI of include/pawsim_b200.h. The driver
 *   - reads the AWSIM key/value parameter file with the reference's defaults, per-key
 *     conversions (strtoul / atoi / strtod), derived flags and validation
 *     (model_code/config.c:42-459), then the grid and time conventions (pawsim.c:126-196);
 *   - reads the raw little-endian float64 data files relative to the parameter file, with
 *     the reference's array orders and defaults (model_code/state.c:67-87, 968-1006;
 *     defs.c:140-426) and, with `restart`, the U/V/H pickup files from the output directory
 *     (state.c:1106-1151);
 *   - runs the preliminary pressure correction, writes the n = 0 state, steps Nt times and
 *     writes U{k}, V{k}, H{k}, W{k} and P on the model-time save schedule
 *     (pawsim.c:318-350; diagnostics.c:84-93, 874-908);
 *   - accumulates the online averages of savefreqAvg and writes each window, and appends
 *     the energy and enstrophy line of savefreqEZ to EZdiags.dat (diagnostics.c:307-700);
 *   - prints "PAWSIM pressure solve" lines and the closing summary when pressureTiming is
 *     set (pawsim.c:100-108, 515-522).
 * Exit status 0 on success, 1 on any failure, with the message on stderr.
 * GPU-only controls come from the environment: PAWSIM_GPU_MG_FP32=1 runs FP32 V-cycles
 * inside FP64 defect correction (PAWSIM_GPU_MG_FP32_INNER of them per defect step); PAWSIM_GPU_SYNC_OUTPUT=1 writes each save before the next
 * step instead of from the background writer (the default: the state is snapshotted on the
 * device and a second thread writes the files while the model steps on).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pawsim_b200.h"

#define NAMELEN 256

/* ------------------------------------------------------------------ configuration */

typedef struct
{
  /* unsigned integers (strtoul) */
  unsigned Nlay, Nx, Ny, Nt, startIdx, timeSteppingScheme, momentumScheme, thicknessScheme,
      tracerScheme, tauNrecs, wDiaNrecs, maxiters, pressureSolver;
  int mpiNx, mpiNy;
  /* booleans (atoi != 0) */
  int useTrad, use_MG, use_fullMG, pressureTiming, writeInitDiagnostics, restart, useWallEW,
      useWallNS, useRL, oceanSurfDrag, windFeedback, useTracer, useBuoyancy, useRandomForcing;
  /* reals (strtod) */
  double Lx, Ly, dt, tmin, tmax, savefrequency, savefreqAvg, savefreqEZ, savefreqUMom, savefreqVMom,
      savefreqThic, savefreqEnergy, savefreqTracer, KT00_sigma, h0, hsml, hmin_surf, hbbl, hmin_bot,
      A2, A4, A2smag, A4smag, K2, K4, linDragCoeff, quadDragCoeff, linDragSurf, quadDragSurf,
      tauPeriod, wDiaPeriod, convDiff, omega_MG, tol, SOR_rp;
  /* derived */
  int useWind, useFbaro, useRelax, useWDia, useDiaVisc;
  double dx, dy;
  char files[32][NAMELEN];
} config;

/* data-file keys, in a fixed order used as indices into config.files */
static const char * FILE_KEYS[] = {
    "hInitFile", "uInitFile", "vInitFile", "bInitFile", "hbFile", "hsFile", "OmegazFile", "gFile",
    "tauxFile", "tauyFile", "uLidFile", "vLidFile", "FbaroXFile", "FbaroYFile", "uRelaxFile",
    "vRelaxFile", "hRelaxFile", "eRelaxFile", "bRelaxFile", "uTimeFile", "vTimeFile", "hTimeFile",
    "eTimeFile", "bTimeFile", "wDiaFile", "diaDiffFile", "diaViscUFile", "diaViscVFile",
    "bFluxFile", NULL};

static int file_index (const char * key)
{
  int i;
  for (i = 0; FILE_KEYS[i]; i ++)
    if (strcmp(FILE_KEYS[i],key) == 0) return i;
  return -1;
}

static const char * file_of (const config * c, const char * key)
{
  int i = file_index(key);
  return (i >= 0) ? c->files[i] : "";
}

/* pawsim_config_defaults (config.c:42-122) */
static void config_defaults (config * c)
{
  memset(c,0,sizeof(*c));
  c->timeSteppingScheme = 5;
  c->momentumScheme = 3;
  c->tmin = -1;
  c->KT00_sigma = 1.4;
  c->tol = 1e-10;
  c->SOR_rp = 1.0;
  c->omega_MG = 2.0 / 3.0;
  c->tauNrecs = 1;
  c->wDiaNrecs = 1;
  c->maxiters = 10000;
  c->useRL = 1;
  c->oceanSurfDrag = 1;
}

typedef enum { K_UINT, K_BOOL, K_SINT, K_REAL } kind;
typedef struct { const char * name; kind k; size_t off; } keydef;

#define U(n) {#n, K_UINT, offsetof(config,n)}
#define B(n) {#n, K_BOOL, offsetof(config,n)}
#define S(n) {#n, K_SINT, offsetof(config,n)}
#define R(n) {#n, K_REAL, offsetof(config,n)}
static const keydef KEYS[] = {
    U(Nlay), U(Nx), U(Ny), U(Nt), U(startIdx), U(timeSteppingScheme), U(momentumScheme),
    U(thicknessScheme), U(tracerScheme), U(tauNrecs), U(wDiaNrecs), U(maxiters), S(mpiNx), S(mpiNy),
    B(useTrad), B(use_MG), B(use_fullMG), B(pressureTiming), B(writeInitDiagnostics), B(restart),
    B(useWallEW), B(useWallNS), B(useRL), B(oceanSurfDrag), B(windFeedback), B(useTracer),
    B(useBuoyancy), B(useRandomForcing), R(Lx), R(Ly), R(dt), R(tmin), R(tmax), R(savefrequency), R(savefreqAvg),
    R(savefreqEZ), R(savefreqUMom), R(savefreqVMom), R(savefreqThic), R(savefreqEnergy), R(savefreqTracer),
    R(KT00_sigma), R(h0), R(hsml), R(hmin_surf), R(hbbl), R(hmin_bot), R(A2), R(A4), R(A2smag),
    R(A4smag), R(K2), R(K4), R(linDragCoeff), R(quadDragCoeff), R(linDragSurf), R(quadDragSurf),
    R(tauPeriod), R(wDiaPeriod), R(convDiff), R(omega_MG), R(tol), {NULL, K_REAL, 0}};
#undef U
#undef B
#undef S
#undef R

/* pawsim_config_read (config.c:129-314): whitespace-separated name/value pairs */
static int config_read (const char * path, config * c)
{
  FILE * fh = fopen(path,"r");
  char key[NAMELEN], val[NAMELEN];
  int solver_given = 0, i;
  if (!fh)
  {
    fprintf(stderr,"Could not open input file %s\n",path);
    return 0;
  }
  while (fscanf(fh,"%255s",key) == 1)
  {
    const keydef * d;
    if (fscanf(fh,"%255s",val) != 1)
    {
      fprintf(stderr,"Missing value for parameter %s\n",key);
      fclose(fh);
      return 0;
    }
    for (d = KEYS; d->name; d ++)
      if (strcmp(d->name,key) == 0) break;
    if (d->name)
    {
      char * p = (char *) c + d->off;
      switch (d->k)
      {
        case K_UINT: *(unsigned *) p = (unsigned) strtoul(val,NULL,10); break;
        case K_BOOL: *(int *) p = atoi(val) != 0; break;
        case K_SINT: *(int *) p = atoi(val); break;
        case K_REAL: *(double *) p = strtod(val,NULL); break;
      }
    }
    else if (strcmp(key,"SOR_rp") == 0 || strcmp(key,"SOR_rp_min") == 0)
      c->SOR_rp = strtod(val,NULL);
    else if (strcmp(key,"pressureSolver") == 0)
    {
      c->pressureSolver = (unsigned) strtoul(val,NULL,10);
      solver_given = 1;
    }
    else if ((i = file_index(key)) >= 0)
    {
      snprintf(c->files[i],NAMELEN,"%s",val);
    }
  }
  fclose(fh);
  /* use_MG and pressureSolver are two spellings of the solver choice (config.c:289-297) */
  if (!solver_given) c->pressureSolver = c->use_MG ? 1 : 0;
  else c->use_MG = c->pressureSolver != 0;
  c->useWind = file_of(c,"tauxFile")[0] || file_of(c,"tauyFile")[0];
  c->useFbaro = file_of(c,"FbaroXFile")[0] || file_of(c,"FbaroYFile")[0];
  c->useRelax = file_of(c,"uTimeFile")[0] || file_of(c,"vTimeFile")[0] || file_of(c,"hTimeFile")[0]
             || file_of(c,"eTimeFile")[0] || (c->useTracer && file_of(c,"bTimeFile")[0]);
  c->useWDia = c->useRelax || file_of(c,"wDiaFile")[0];
  c->useDiaVisc = file_of(c,"diaViscUFile")[0] || file_of(c,"diaViscVFile")[0] || c->convDiff != 0;
  return 1;
}

/* pawsim_config_validate (config.c:320-459) */
static int config_validate (const config * c)
{
  const char * msg = NULL;
  if (c->Nlay == 0 || c->Nx == 0 || c->Ny == 0) msg = "Nlay, Nx and Ny must all be specified and positive";
  else if (c->Ly <= 0) msg = "Ly must be specified and positive";
  else if (c->timeSteppingScheme > 5 || c->momentumScheme > 3 || c->thicknessScheme > 3 || c->tracerScheme > 2)
    msg = "Unknown or unsupported numerical scheme identifier";
  else if (c->h0 < 0) msg = "h0 must be non-negative";
  else if (c->hsml < 0 || c->hmin_surf < 0 || c->hbbl < 0 || c->hmin_bot < 0 || c->linDragCoeff < 0
           || c->quadDragCoeff < 0 || c->linDragSurf < 0 || c->quadDragSurf < 0 || c->A2 < 0 || c->A4 < 0
           || c->A2smag < 0 || c->A4smag < 0 || c->K2 < 0 || c->K4 < 0 || c->convDiff < 0
           || c->tauNrecs == 0 || c->wDiaNrecs == 0)
    msg = "Invalid wind forcing parameters";
  else if (c->tol <= 0 || c->SOR_rp <= 0 || c->SOR_rp >= 2 || c->omega_MG <= 0 || c->maxiters == 0)
    msg = "Invalid pressure solver parameters";
  else if (c->pressureSolver > 2) msg = "Unknown pressureSolver identifier";
  else if ((c->mpiNx == 0 || c->mpiNy == 0) && (c->mpiNx != 0 || c->mpiNy != 0))
    msg = "mpiNx and mpiNy must both be specified or both omitted";
  else if (c->mpiNx < 0 || c->mpiNy < 0) msg = "mpiNx and mpiNy must be non-negative";
  else if (c->useBuoyancy && !c->useTracer) msg = "useBuoyancy requires useTracer in PAWSIM";
  else if (c->useTrad) msg = "AWSIM useTrad time stepping is not ported in PAWSIM";
  else if (c->useRandomForcing)
    msg = "AWSIM random forcing is not ported in PAWSIM; prescribe deterministic forcing instead";
  else if (c->timeSteppingScheme < 3) msg = "PAWSIM only supports AB1, AB2 and AB3 time stepping so far";
  if (msg)
  {
    fprintf(stderr,"%s\n",msg);
    return 0;
  }
  return 1;
}

/* setGridDimensions and setTimeParameters (pawsim.c:126-196) */
static int grid_and_time (config * c)
{
  int cnt;
  if (c->Lx <= 0) c->Lx = c->Ly * c->Nx / c->Ny;
  c->dx = c->Lx / c->Nx;
  c->dy = c->Ly / c->Ny;
  cnt = (c->Nt > 0) + (c->tmax > 0) + (c->dt > 0);
  if (cnt != 2)
  {
    fprintf(stderr,"Must specify exactly two of {Nt, tmax, dt}\n");
    return 0;
  }
  if (c->tmin < 0) c->tmin = c->restart ? c->startIdx * c->savefrequency : 0;
  if (c->Nt == 0)
  {
    if (c->tmax <= c->tmin)
    {
      fprintf(stderr,"Integration end time must exceed integration start time\n");
      return 0;
    }
    c->Nt = (unsigned) ceil((c->tmax - c->tmin) / c->dt);
  }
  if (c->dt == 0)
  {
    if (c->tmax <= c->tmin)
    {
      fprintf(stderr,"Integration end time must exceed integration start time\n");
      return 0;
    }
    c->dt = (c->tmax - c->tmin) / c->Nt;
  }
  if (c->savefrequency == 0) c->savefrequency = c->dt;
  if (c->tmax == 0) c->tmax = c->tmin + c->dt * c->Nt;
  if (c->tmin >= c->tmax)
  {
    fprintf(stderr,"Integration start time exceeds integration end time\n");
    return 0;
  }
  return 1;
}

/* ------------------------------------------------------------------ data files */

static char g_indir[4096] = ".";

/* paths are relative to the parameter file's directory unless absolute (state.c:67-87) */
static void resolve (const char * name, char * out, size_t n)
{
  if (name[0] == '/') snprintf(out,n,"%s",name);
  else snprintf(out,n,"%s/%s",g_indir,name);
}

/* raw little-endian float64 values (the hosts this runs on are little-endian) */
static int read_f64 (const char * path, double * dst, size_t n)
{
  FILE * fh = fopen(path,"rb");
  size_t got;
  if (!fh)
  {
    fprintf(stderr,"Could not open %s\n",path);
    return 0;
  }
  got = fread(dst,sizeof(double),n,fh);
  fclose(fh);
  if (got < n)
  {
    fprintf(stderr,"Could only read %zu of %zu values from %s\n",got,n,path);
    return 0;
  }
  return 1;
}

static int write_f64 (const char * outdir, const char * name, const double * src, size_t n)
{
  char path[8192];
  FILE * fh;
  size_t len = strlen(outdir);
  snprintf(path,sizeof(path),"%s%s%s",outdir,(len > 0 && outdir[len - 1] != '/') ? "/" : "",name);
  fh = fopen(path,"wb");
  if (!fh)
  {
    fprintf(stderr,"Could not open %s for writing\n",path);
    return 0;
  }
  if (fwrite(src,sizeof(double),n,fh) != n)
  {
    fclose(fh);
    fprintf(stderr,"Could not write %s\n",path);
    return 0;
  }
  fclose(fh);
  return 1;
}

/* ------------------------------------------------------------------ model set-up */

static int gpu_ok (int rc, const char * what)
{
  if (rc < 0)
  {
    fprintf(stderr,"ERROR: %s: %s\n",what,pawsim_gpu_last_error());
    return 0;
  }
  return 1;
}

static void fill (double * a, size_t n, double v)
{
  size_t q;
  for (q = 0; q < n; q ++) a[q] = v;
}

/* upload one 2-D field (Ny x Nx, x fastest) */
static int put (pawsim_gpu * m, const char * name, int k, const double * a, size_t n)
{
  return gpu_ok(pawsim_gpu_set_field(m,name,k,a,n),name);
}

/* a 3-D AWSIM file (layer fastest, then x, then y) split into L planes (Ny x Nx) */
static int put_layers (pawsim_gpu * m, const config * c, const char * key, const char * name, double deflt,
                       int deflt_eta, double * plane, double * buf)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  const unsigned L = c->Nlay;
  unsigned k;
  const char * f = file_of(c,key);
  char path[8192];
  if (f[0])
  {
    resolve(f,path,sizeof(path));
    if (!read_f64(path,buf,N * L)) return 0;
  }
  for (k = 0; k < L; k ++)
  {
    size_t q;
    if (f[0])
      for (q = 0; q < N; q ++) plane[q] = buf[q * L + k];
    else
      fill(plane,N,deflt_eta ? 1000.0 * k / L : deflt);
    if (!put(m,name,(int) k,plane,N)) return 0;
  }
  return 1;
}

static int put_plane (pawsim_gpu * m, const config * c, const char * key, const char * name, double deflt,
                      double * plane)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  const char * f = file_of(c,key);
  char path[8192];
  if (f[0])
  {
    resolve(f,path,sizeof(path));
    if (!read_f64(path,plane,N)) return 0;
  }
  else
    fill(plane,N,deflt);
  return put(m,name,0,plane,N);
}

static int upload_inputs (pawsim_gpu * m, const config * c, const char * outdir)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  const unsigned L = c->Nlay, nt = c->tauNrecs, nw = c->wDiaNrecs;
  size_t big = N * (size_t) (L + 1) * (nt > nw ? nt : nw) + (size_t) (c->Nx + 1) * (c->Ny + 1);
  double * buf = malloc(big * sizeof(double));
  double * plane = malloc(((size_t) (c->Nx + 1) * (c->Ny + 1)) * sizeof(double));
  char path[8192];
  int ok = buf && plane;
  unsigned k, r;
  const char * f;
  /* prognostic initial state and the restoring/viscosity layer fields (state.c:968-1006) */
  ok = ok && put_layers(m,c,"uInitFile","u",0,0,plane,buf) && put_layers(m,c,"vInitFile","v",0,0,plane,buf)
          && put_layers(m,c,"hInitFile","h",0,0,plane,buf)
          && put_layers(m,c,"uRelaxFile","uRelax",0,0,plane,buf)
          && put_layers(m,c,"vRelaxFile","vRelax",0,0,plane,buf)
          && put_layers(m,c,"hRelaxFile","hRelax",1000.0 / L,0,plane,buf)
          && put_layers(m,c,"eRelaxFile","eRelax",0,1,plane,buf)
          && put_layers(m,c,"uTimeFile","uTime",-1,0,plane,buf)
          && put_layers(m,c,"vTimeFile","vTime",-1,0,plane,buf)
          && put_layers(m,c,"eTimeFile","eTime",-1,0,plane,buf)
          && put_layers(m,c,"diaViscUFile","nu_u_dia",0,0,plane,buf)
          && put_layers(m,c,"diaViscVFile","nu_v_dia",0,0,plane,buf);
  if (c->useTracer)   /* tracer state and restoring (state.c:968-1006: b 0, bRelax 0, bTime -1) */
    ok = ok && put_layers(m,c,"bInitFile","b",0,0,plane,buf) && put_layers(m,c,"bRelaxFile","bRelax",0,0,plane,buf)
            && put_layers(m,c,"bTimeFile","bTime",-1,0,plane,buf)
            && put_layers(m,c,"diaDiffFile","kappa_dia",0,0,plane,buf)
            && put_plane(m,c,"bFluxFile","Fsurf_b",0,plane);
  ok = ok && put_plane(m,c,"hsFile","hhs",0,plane) && put_plane(m,c,"hbFile","hhb",0,plane)
          && put_plane(m,c,"uLidFile","uLid",0,plane) && put_plane(m,c,"vLidFile","vLid",0,plane)
          && put_plane(m,c,"FbaroXFile","Fbaro_x",0,plane) && put_plane(m,c,"FbaroYFile","Fbaro_y",0,plane)
          && put_plane(m,c,"hTimeFile","hTime",-1,plane);
  /* planetary vorticity on the (Nx+1) x (Ny+1) q grid */
  if (ok)
  {
    const size_t NQ = (size_t) (c->Nx + 1) * (c->Ny + 1);
    f = file_of(c,"OmegazFile");
    if (f[0])
    {
      resolve(f,path,sizeof(path));
      ok = read_f64(path,plane,NQ);
    }
    else
      fill(plane,NQ,0);
    ok = ok && put(m,"omegaz",0,plane,NQ);
  }
  /* gravities */
  if (ok)
  {
    f = file_of(c,"gFile");
    if (f[0])
    {
      resolve(f,path,sizeof(path));
      ok = read_f64(path,plane,L);
      for (k = 0; ok && k < L; k ++)
        if (plane[k] < 0)
        {
          fprintf(stderr,"gFile may contain only non-negative values\n");
          ok = 0;
        }
    }
    else
      fill(plane,L,9.81);
    ok = ok && put(m,"gg",0,plane,L);
  }
  /* wind records (record fastest, then x, then y) */
  {
    const char * keys[2] = {"tauxFile","tauyFile"};
    const char * names[2] = {"taux","tauy"};
    int a;
    for (a = 0; ok && a < 2; a ++)
    {
      f = file_of(c,keys[a]);
      if (f[0])
      {
        resolve(f,path,sizeof(path));
        ok = read_f64(path,buf,N * nt);
      }
      for (r = 0; ok && r < nt; r ++)
      {
        size_t q;
        if (f[0])
          for (q = 0; q < N; q ++) plane[q] = buf[q * nt + r];
        else
          fill(plane,N,0);
        ok = put(m,names[a],(int) r,plane,N);
      }
    }
  }
  /* diapycnal velocity records (record fastest, then interface, then x, then y) */
  if (ok)
  {
    f = file_of(c,"wDiaFile");
    if (f[0])
    {
      resolve(f,path,sizeof(path));
      ok = read_f64(path,buf,N * (L + 1) * nw);
    }
    for (r = 0; ok && r < nw; r ++)
      for (k = 0; ok && k <= L; k ++)
      {
        size_t q;
        if (f[0])
          for (q = 0; q < N; q ++) plane[q] = buf[(q * (L + 1) + k) * nw + r];
        else
          fill(plane,N,0);
        ok = put(m,"wdia_ff",(int) (r * (L + 1) + k),plane,N);
      }
  }
  /* restart: the U/V/H pickup files of the output directory (state.c:1106-1151) */
  if (ok && c->restart)
  {
    const char * pre[4] = {"U","V","H","B"};
    const char * nm[4] = {"u","v","h","b"};
    int a;
    for (k = 0; ok && k < L; k ++)
      for (a = 0; ok && a < (c->useTracer ? 4 : 3); a ++)
      {
        snprintf(path,sizeof(path),"%s/%s%u_n=%u.dat",outdir,pre[a],k,c->startIdx);
        ok = read_f64(path,plane,N) && put(m,nm[a],(int) k,plane,N);
      }
  }
  free(buf);
  free(plane);
  return ok;
}

/* pawsim_diagnostics_write_model_state (diagnostics.c:874-908) */
static int write_state (pawsim_gpu * m, const config * c, const char * outdir, unsigned n, double * plane)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  char name[NAMELEN];
  unsigned k;
  const char * pre[4] = {"U","V","H","B"};
  const char * nm[4] = {"u","v","h","b"};
  int a;
  for (k = 0; k < c->Nlay; k ++)
  {
    for (a = 0; a < (c->useTracer ? 4 : 3); a ++)
    {
      snprintf(name,sizeof(name),"%s%u_n=%u.dat",pre[a],k,n);
      if (!gpu_ok(pawsim_gpu_get_field(m,nm[a],(int) k,plane,N),nm[a]) || !write_f64(outdir,name,plane,N))
        return 0;
    }
    snprintf(name,sizeof(name),"W%u_n=%u.dat",k,n);
    if (!gpu_ok(pawsim_gpu_get_field(m,"wdia",(int) k,plane,N),"wdia") || !write_f64(outdir,name,plane,N))
      return 0;
  }
  snprintf(name,sizeof(name),"W%u_n=%u.dat",c->Nlay,n);
  if (!gpu_ok(pawsim_gpu_get_field(m,"wdia",(int) c->Nlay,plane,N),"wdia") || !write_f64(outdir,name,plane,N))
    return 0;
  if (c->useRL)
  {
    snprintf(name,sizeof(name),"P_n=%u.dat",n);
    if (!gpu_ok(pawsim_gpu_get_field(m,"pi",0,plane,N),"pi") || !write_f64(outdir,name,plane,N)) return 0;
  }
  return 1;
}

/* the files of one save from the planes of pawsim_gpu_save_begin (u, v, h, b per layer,
 * w_dia per interface, pi), under the names of write_state */
static int write_save_planes (const config * c, const char * outdir, unsigned n, const double * host)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  const char * pre[4] = {"U","V","H","B"};
  char name[NAMELEN];
  unsigned k;
  int a;
  for (k = 0; k < c->Nlay; k ++)
  {
    for (a = 0; a < (c->useTracer ? 4 : 3); a ++)
    {
      snprintf(name,sizeof(name),"%s%u_n=%u.dat",pre[a],k,n);
      if (!write_f64(outdir,name,host,N)) return 0;
      host += N;
    }
  }
  for (k = 0; k <= c->Nlay; k ++)
  {
    snprintf(name,sizeof(name),"W%u_n=%u.dat",k,n);
    if (!write_f64(outdir,name,host,N)) return 0;
    host += N;
  }
  if (c->useRL)
  {
    snprintf(name,sizeof(name),"P_n=%u.dat",n);
    if (!write_f64(outdir,name,host,N)) return 0;
  }
  return 1;
}

/* Background writer of the asynchronous saves: the main loop snapshots the state with
 * pawsim_gpu_save_begin and queues (slot, n); this thread waits for the slot's host copy,
 * writes that save's files and releases the slot, while the model steps on. */
typedef struct
{
  pawsim_gpu * m;
  const config * c;
  const char * outdir;
  pthread_t th;
  pthread_mutex_t mu;
  pthread_cond_t cv;
  int slot[2];
  unsigned n[2];
  int head, count, stop, failed;
} writer;

static void * writer_main (void * arg)
{
  writer * w = (writer *) arg;
  for (;;)
  {
    int slot, ok;
    unsigned n;
    const double * host = NULL;
    pthread_mutex_lock(&w->mu);
    while (w->count == 0 && !w->stop) pthread_cond_wait(&w->cv,&w->mu);
    if (w->count == 0)
    {
      pthread_mutex_unlock(&w->mu);
      break;
    }
    slot = w->slot[w->head];
    n = w->n[w->head];
    pthread_mutex_unlock(&w->mu);
    ok = gpu_ok(pawsim_gpu_save_wait(w->m,slot,&host),"save") && write_save_planes(w->c,w->outdir,n,host);
    if (!ok) fprintf(stderr,"Unable to write model state n=%u\n",n);
    pawsim_gpu_save_release(w->m,slot);
    pthread_mutex_lock(&w->mu);
    w->head = (w->head + 1) % 2;
    w->count --;
    if (!ok) w->failed = 1;
    pthread_cond_broadcast(&w->cv);
    pthread_mutex_unlock(&w->mu);
  }
  return NULL;
}

static int writer_start (writer * w, pawsim_gpu * m, const config * c, const char * outdir)
{
  memset(w,0,sizeof(*w));
  w->m = m;
  w->c = c;
  w->outdir = outdir;
  pthread_mutex_init(&w->mu,NULL);
  pthread_cond_init(&w->cv,NULL);
  if (pthread_create(&w->th,NULL,writer_main,w) != 0)
  {
    fprintf(stderr,"ERROR: could not start the output thread\n");
    return 0;
  }
  return 1;
}

/* snapshot the current state as save n and queue its files */
static int writer_push (writer * w, unsigned n)
{
  int slot, failed;
  pthread_mutex_lock(&w->mu);
  failed = w->failed;
  pthread_mutex_unlock(&w->mu);
  if (failed || !gpu_ok(pawsim_gpu_save_begin(w->m,&slot),"save")) return 0;
  pthread_mutex_lock(&w->mu);
  while (w->count == 2) pthread_cond_wait(&w->cv,&w->mu);
  w->slot[(w->head + w->count) % 2] = slot;
  w->n[(w->head + w->count) % 2] = n;
  w->count ++;
  pthread_cond_broadcast(&w->cv);
  pthread_mutex_unlock(&w->mu);
  return 1;
}

/* write what is queued, stop the thread; 0 if any save failed */
static int writer_finish (writer * w)
{
  int failed;
  pthread_mutex_lock(&w->mu);
  w->stop = 1;
  pthread_cond_broadcast(&w->cv);
  pthread_mutex_unlock(&w->mu);
  pthread_join(w->th,NULL);
  failed = w->failed;
  pthread_mutex_destroy(&w->mu);
  pthread_cond_destroy(&w->cv);
  return !failed;
}

/* one completed online-average window under AWSIM's names (diagnostics.c:378-420) */
static int write_averages (pawsim_gpu * m, const config * c, const char * outdir, unsigned n, double * plane)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  const char * nm[10] = {"U_avg","V_avg","H_avg","M_avg","W_avg","HU_avg","HV_avg","HUU_avg","HVV_avg","HUV_avg"};
  char name[NAMELEN];
  unsigned k;
  int a;
  for (k = 0; k < c->Nlay; k ++)
  {
    for (a = 0; a < 10; a ++)
    {
      snprintf(name,sizeof(name),"%s%u_n=%u.dat",nm[a],k,n);
      if (!gpu_ok(pawsim_gpu_get_field(m,nm[a],(int) k,plane,N),nm[a]) || !write_f64(outdir,name,plane,N)) return 0;
    }
    if (c->useTracer)
    {
      snprintf(name,sizeof(name),"B_avg%u_n=%u.dat",k,n);
      if (!gpu_ok(pawsim_gpu_get_field(m,"B_avg",(int) k,plane,N),"B_avg") || !write_f64(outdir,name,plane,N)) return 0;
    }
  }
  snprintf(name,sizeof(name),"W_avg%u_n=%u.dat",c->Nlay,n);
  if (!gpu_ok(pawsim_gpu_get_field(m,"W_avg",(int) c->Nlay,plane,N),"W_avg") || !write_f64(outdir,name,plane,N))
    return 0;
  if (c->useRL)
  {
    snprintf(name,sizeof(name),"P_avg_n=%u.dat",n);
    if (!gpu_ok(pawsim_gpu_get_field(m,"P_avg",0,plane,N),"P_avg") || !write_f64(outdir,name,plane,N)) return 0;
  }
  return 1;
}

/* every EZdiags.dat line now due (diagnostics.c:478-700): the time of the line, KE, PE,
 * KE+PE and the enstrophy of each layer, all from the current state */
static int write_ez (pawsim_gpu * m, const config * c, const char * outdir, double t, unsigned * n_EZ,
                     double * t_next_EZ)
{
  char path[8192];
  double KE, PE, Z[8];
  size_t len = strlen(outdir);
  unsigned k;
  /* the reference builds eta from the thickness last copied into its work arrays: the
   * pressure RHS (rigid lid) and the online averages copy the current state; otherwise the
   * last tendency evaluation copied the state of the start of the step */
  int eta_prev = !c->useRL && !(c->savefreqAvg > 0);
  if (!gpu_ok(pawsim_gpu_energy(m,eta_prev,&KE,&PE,Z),"energy diagnostics")) return 0;
  snprintf(path,sizeof(path),"%s%sEZdiags.dat",outdir,(len > 0 && outdir[len - 1] != '/') ? "/" : "");
  while (t >= *t_next_EZ)
  {
    FILE * fh = fopen(path,(c->restart || *n_EZ > 1) ? "a" : "w");
    if (!fh)
    {
      fprintf(stderr,"Could not open %s for writing\n",path);
      return 0;
    }
    fprintf(fh,"%le",*t_next_EZ);
    fprintf(fh," %.50e %.50e %.50e ",KE,PE,KE + PE);
    for (k = 0; k < c->Nlay; k ++) fprintf(fh,"%.50e ",Z[k]);
    fprintf(fh,"\n");
    fclose(fh);
    (*n_EZ) ++;
    *t_next_EZ = *n_EZ * c->savefreqEZ;
  }
  return 1;
}

/* budget families (config bit f) and their output names (diagnostics.c:758-796) */
static const char * const BUDGET_NAMES[5][16] = {
  {"UMom_PVadvection","UMom_Montgomery","UMom_KEgradient","UMom_dhdt","UMom_viscosity","UMom_hypervisc",
   "UMom_linBotDrag","UMom_linSurfDrag","UMom_quadBotDrag","UMom_quadSurfDrag","UMom_windStress",
   "UMom_buoyForce","UMom_relaxation","UMom_diapycnal","UMom_baroForcing","UMom_diaVisc"},
  {"VMom_PVadvection","VMom_Montgomery","VMom_KEgradient","VMom_dhdt","VMom_viscosity","VMom_hypervisc",
   "VMom_linBotDrag","VMom_linSurfDrag","VMom_quadBotDrag","VMom_quadSurfDrag","VMom_windStress",
   "VMom_buoyForce","VMom_relaxation","VMom_diapycnal","VMom_baroForcing","VMom_diaVisc"},
  {"Thic_advection","Thic_relaxation"},
  {"Energy_advection","Energy_Montgomery","Energy_windStress","Energy_linBotDrag","Energy_linSurfDrag",
   "Energy_quadBotDrag","Energy_quadSurfDrag","Energy_viscosity","Energy_hypervisc","Energy_diaProd",
   "Energy_diaAdv","Energy_baroForcing","Energy_buoyForce","Energy_relaxation","Energy_diaVisc"},
  {"Tracer_advection","Tracer_diaAdv","Tracer_isoDiff","Tracer_hyperdiff","Tracer_diaDiff","Tracer_relaxation"}};
static const unsigned BUDGET_TERMS[5] = {16,16,2,15,6};

/* one family's window (diagnostics.c:798-864): sums / ((n - n_prev) dt), written, reset */
static int write_budget (pawsim_gpu * m, const config * c, const char * outdir, int f, unsigned n,
                         unsigned n_prev, unsigned n_out, double * plane)
{
  const size_t N = (size_t) c->Nx * c->Ny;
  char name[NAMELEN];
  unsigned t, k;
  double len = (n - n_prev) * c->dt;
  if (!gpu_ok(pawsim_gpu_scale_budgets(m,1 << f,1 / len),"budgets")) return 0;
  for (t = 0; t < BUDGET_TERMS[f]; t ++)
  {
    for (k = 0; k < c->Nlay; k ++)
    {
      snprintf(name,sizeof(name),"%s%u_n=%u.dat",BUDGET_NAMES[f][t],k,n_out);
      if (!gpu_ok(pawsim_gpu_get_field(m,BUDGET_NAMES[f][t],(int) k,plane,N),"budgets")
       || !write_f64(outdir,name,plane,N)) return 0;
    }
  }
  return gpu_ok(pawsim_gpu_zero_budgets(m,1 << f),"budgets");
}

static const char * solver_name (unsigned s)
{
  return s == 0 ? "SOR" : (s == 1 ? "MG_GATHERED" : (s == 2 ? "MG_DISTRIBUTED" : "UNKNOWN"));
}

int main (int argc, char ** argv)
{
  config c;
  pawsim_gpu_config g;
  pawsim_gpu * m = NULL;
  pawsim_gpu_stats st;
  const char * outdir;
  double * plane = NULL;
  unsigned n, n_saves, solves = 0, fallbacks = 0, n_avg = 0, n_EZ = 0;
  double t_next_avg = 0, t_next_EZ = 0;
  double bfreq[5];
  unsigned b_out[5] = {0,0,0,0,0}, b_prev[5] = {0,0,0,0,0};
  double b_next[5] = {0,0,0,0,0};
  int f;
  double wall_total = 0, iters_total = 0;
  const char * slash;
  int rc = 1;
  writer wr;
  int async_out = !(getenv("PAWSIM_GPU_SYNC_OUTPUT") && atoi(getenv("PAWSIM_GPU_SYNC_OUTPUT")));
  int writer_on = 0;

  if (argc < 3)
  {
    fprintf(stderr,"Usage: PAWSIM_B200.exe <input_file> <output_dir>\n");
    return 1;
  }
  outdir = argv[2];
  slash = strrchr(argv[1],'/');
  if (slash)
  {
    size_t len = (size_t) (slash - argv[1]);
    if (len >= sizeof(g_indir)) len = sizeof(g_indir) - 1;
    memcpy(g_indir,argv[1],len);
    g_indir[len] = '\0';
  }
  config_defaults(&c);
  if (!config_read(argv[1],&c) || !config_validate(&c) || !grid_and_time(&c)) return 1;

  memset(&g,0,sizeof(g));
  g.Nx = (int) c.Nx;
  g.Ny = (int) c.Ny;
  g.Nlay = (int) c.Nlay;
  g.wall_ew = c.useWallEW;
  g.wall_ns = c.useWallNS;
  g.ts_scheme = (int) c.timeSteppingScheme;
  g.mom_scheme = (int) c.momentumScheme;
  g.thick_scheme = (int) c.thicknessScheme;
  g.use_rl = c.useRL;
  g.ocean_surf_drag = c.oceanSurfDrag;
  g.wind_feedback = c.windFeedback;
  g.use_wind = c.useWind;
  g.use_fbaro = c.useFbaro;
  g.use_relax = c.useRelax;
  g.use_wdia = c.useWDia;
  g.use_diavisc = c.useDiaVisc;
  g.use_wdia_file = file_of(&c,"wDiaFile")[0] != 0;
  g.tau_nrecs = (int) c.tauNrecs;
  g.wdia_nrecs = (int) c.wDiaNrecs;
  g.solver = (int) c.pressureSolver;
  g.use_full_mg = c.use_fullMG;
  g.maxiters = (int) c.maxiters;
  g.pressure_timing = c.pressureTiming;
  g.Lx = c.Lx; g.Ly = c.Ly; g.dt = c.dt; g.tmin = c.tmin;
  g.A2 = c.A2; g.A4 = c.A4; g.A2smag = c.A2smag; g.A4smag = c.A4smag;
  g.h0 = c.h0; g.hsml = c.hsml; g.hmin_surf = c.hmin_surf; g.hbbl = c.hbbl; g.hmin_bot = c.hmin_bot;
  g.KT00_sigma = c.KT00_sigma;
  g.lin_drag = c.linDragCoeff; g.quad_drag = c.quadDragCoeff;
  g.lin_drag_surf = c.linDragSurf; g.quad_drag_surf = c.quadDragSurf;
  g.tau_period = c.tauPeriod; g.wdia_period = c.wDiaPeriod; g.conv_diff = c.convDiff;
  g.pi_tol = c.tol; g.sor_rp = c.SOR_rp; g.omega_mg = c.omega_MG;
  g.mg_fp32 = getenv("PAWSIM_GPU_MG_FP32") ? atoi(getenv("PAWSIM_GPU_MG_FP32")) : 0;
  g.mg_fp32_inner = getenv("PAWSIM_GPU_MG_FP32_INNER") ? atoi(getenv("PAWSIM_GPU_MG_FP32_INNER")) : 0;
  g.mg_pre = 1; g.mg_post = 1; g.mg_omega = -1.0;   /* weight chosen by the solver */
  g.serial_sums = -1;
  g.mg_tile = 0;
  g.use_tracer = c.useTracer;
  g.tracer_scheme = (int) c.tracerScheme;
  g.K2 = c.K2; g.K4 = c.K4;
  g.budgets = (c.savefreqUMom > 0 ? 1 : 0) | (c.savefreqVMom > 0 ? 2 : 0) | (c.savefreqThic > 0 ? 4 : 0)
            | (c.savefreqEnergy > 0 ? 8 : 0) | (c.savefreqTracer > 0 ? 16 : 0);
  g.use_buoyancy = c.useTracer && c.useBuoyancy;
  /* useDiaDiff (config.c:309-310) */
  g.use_diadiff = c.useTracer && (file_of(&c,"diaDiffFile")[0] || file_of(&c,"bFluxFile")[0] || c.convDiff != 0);

  if (!gpu_ok(pawsim_gpu_create(&g,&m),"pawsim_gpu_create")) return 1;
  plane = malloc(((size_t) (c.Nx + 1) * (c.Ny + 1) + c.Nlay + 1) * sizeof(double));
  if (!plane || !upload_inputs(m,&c,outdir) || !gpu_ok(pawsim_gpu_init(m),"pawsim_gpu_init")) goto done;
  printf("PAWSIM parsed %u x %u x %u AWSIM input\n",c.Nx,c.Ny,c.Nlay);
  fflush(stdout);

  n_saves = c.restart ? c.startIdx : 0;
  if (c.savefreqAvg > 0)
  {
    /* restarted runs continue AWSIM's diagnostic numbering (pawsim.c:428-433) */
    n_avg = (unsigned) round(c.tmin / c.savefreqAvg) + 1;
    t_next_avg = c.tmin + c.savefreqAvg;
  }
  if (c.savefreqEZ > 0)
  {
    n_EZ = (unsigned) round(c.tmin / c.savefreqEZ) + 1;
    t_next_EZ = c.tmin + c.savefreqEZ;
  }
  bfreq[0] = c.savefreqUMom; bfreq[1] = c.savefreqVMom; bfreq[2] = c.savefreqThic;
  bfreq[3] = c.savefreqEnergy; bfreq[4] = c.useTracer ? c.savefreqTracer : 0;
  for (f = 0; f < 5; f ++)
  {
    if (bfreq[f] > 0)
    {
      b_out[f] = (unsigned) round(c.tmin / bfreq[f]) + 1;
      b_next[f] = c.tmin + bfreq[f];
    }
  }
  /* preliminary rigid-lid correction, then the n = 0 (or pickup) state (pawsim.c:278-312) */
  memset(&st,0,sizeof(st));
  if (!gpu_ok(pawsim_gpu_prelim(m,&st),"preliminary pressure correction")) goto done;
  if (c.useRL)
  {
    solves ++;
    wall_total += st.solve_ms / 1e3;
    iters_total += st.iters;
    fallbacks += st.fallback != 0;
    if (c.pressureTiming)
    {
      printf("PAWSIM pressure solve: phase=prelim n=0 solver=%s",st.fallback ? "MG_GATHERED" : solver_name(c.pressureSolver));
      if (st.fallback) printf(" requested=%s fallback=1",solver_name(c.pressureSolver));
      printf(" iters=%u walltime=%0.6f s residual_max=%0.6e residual_rms=%0.6e div_max=%0.6e div_rms=%0.6e\n",
             (unsigned) st.iters,st.solve_ms / 1e3,st.residual_max,st.residual_rms,st.div_max,st.div_rms);
    }
    printf("PAWSIM pressure iterations: %u\n",(unsigned) st.iters);
    fflush(stdout);
  }
  if (async_out)
  {
    if (!writer_start(&wr,m,&c,outdir)) goto done;
    writer_on = 1;
  }
  if (!(async_out ? writer_push(&wr,n_saves) : write_state(m,&c,outdir,n_saves,plane))) goto done;
  n_saves ++;

  for (n = 1; n <= c.Nt; n ++)
  {
    double t, eps = 1e-9 * fabs(c.dt);
    memset(&st,0,sizeof(st));
    if (!gpu_ok(pawsim_gpu_step(m,n,&st),"time step"))
    {
      fprintf(stderr,"ERROR: PAWSIM time step failed at n=%u\n",n);
      goto done;
    }
    if (c.useRL)
    {
      solves ++;
      wall_total += st.solve_ms / 1e3;
      iters_total += st.iters;
      fallbacks += st.fallback != 0;
      if (c.pressureTiming)
      {
        printf("PAWSIM pressure solve: phase=step n=%u solver=%s",n,
               st.fallback ? "MG_GATHERED" : solver_name(c.pressureSolver));
        if (st.fallback) printf(" requested=%s fallback=1",solver_name(c.pressureSolver));
        printf(" iters=%u walltime=%0.6f s residual_max=%0.6e residual_rms=%0.6e div_max=%0.6e div_rms=%0.6e\n",
               (unsigned) st.iters,st.solve_ms / 1e3,st.residual_max,st.residual_rms,st.div_max,st.div_rms);
        fflush(stdout);
      }
      if ((unsigned) st.iters == c.maxiters)
        fprintf(stderr,"WARNING: PAWSIM pressure solve reached maxiters at n=%u\n",n);
    }
    /* every save whose model time has been reached (pawsim.c:318-350) */
    t = pawsim_gpu_time(m);
    while (c.savefrequency > 0 && !(t + eps < n_saves * c.savefrequency))
    {
      if (!(async_out ? writer_push(&wr,n_saves) : write_state(m,&c,outdir,n_saves,plane)))
      {
        fprintf(stderr,"Unable to write model state n=%u\n",n_saves);
        goto done;
      }
      n_saves ++;
    }
    /* online averages (diagnostics.c:307-470): the step that crosses the window's end adds
     * only its share, then the window is normalised, written and reset */
    if (c.savefreqAvg > 0)
    {
      double avg_fac = (t < t_next_avg) ? 1 : 1 - (t - t_next_avg) / c.dt;
      if (!gpu_ok(pawsim_gpu_accumulate_averages(m,avg_fac),"averages")) goto done;
      if (!(t < t_next_avg))
      {
        if (!gpu_ok(pawsim_gpu_scale_averages(m,1 / c.savefreqAvg),"averages")
         || !write_averages(m,&c,outdir,n_avg,plane)
         || !gpu_ok(pawsim_gpu_zero_averages(m),"averages"))
        {
          fprintf(stderr,"ERROR: PAWSIM diagnostic averaging failed at n=%u\n",n);
          goto done;
        }
        n_avg ++;
        t_next_avg = n_avg * c.savefreqAvg;
      }
    }
    if (c.savefreqEZ > 0 && t >= t_next_EZ && !write_ez(m,&c,outdir,t,&n_EZ,&t_next_EZ))
    {
      fprintf(stderr,"ERROR: PAWSIM diagnostic averaging failed at n=%u\n",n);
      goto done;
    }
    /* budget windows, each family on its own clock (diagnostics.c:756-866) */
    for (f = 0; f < 5; f ++)
    {
      if (bfreq[f] > 0 && t >= b_next[f])
      {
        if (!write_budget(m,&c,outdir,f,n,b_prev[f],b_out[f],plane))
        {
          fprintf(stderr,"ERROR: PAWSIM diagnostic averaging failed at n=%u\n",n);
          goto done;
        }
        b_prev[f] = n;
        b_out[f] ++;
        b_next[f] = b_out[f] * bfreq[f];
      }
    }
  }
  if (c.pressureTiming && solves > 0)
  {
    printf("PAWSIM pressure summary: requested=%s solves=%u fallback_solves=%u total_walltime=%0.6f s "
           "mean_walltime=%0.6f s mean_iters=%0.2f\n",
           solver_name(c.pressureSolver),solves,fallbacks,wall_total,wall_total / solves,iters_total / solves);
    fflush(stdout);
  }
  rc = 0;
done:
  if (writer_on && !writer_finish(&wr)) rc = 1;
  free(plane);
  pawsim_gpu_destroy(m);
  return rc;
}
