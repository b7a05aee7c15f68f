/*
 * ref_harness.c -- times the reference's own serial hot path, step by step.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU baseline of bench.py and a pinning aid). Linked
 * against the reference's objects built from their sources by oracle/Makefile; it calls
 * the reference's public functions in the order of model_code/pawsim.c:355-511 (without
 * output files or diagnostics) and prints one JSON line per timed phase:
 *
 *   ref_harness <param_file> <nsteps> [state_out_prefix]
 *
 * Grid and time set-up repeat pawsim.c:126-196 (those helpers are static there).
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "context.h"
#include "integrator.h"
#include "forcing.h"
#include "pressure.h"
#include "tendency.h"

static double now (void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC,&ts);
  return ts.tv_sec + 1e-9*ts.tv_nsec;
}

static int dump (const char * prefix, const char * name, int k, pawsim_field2d * f)
{
  char path[1024];
  FILE * fp;
  uint i,j,g = f->nghost;
  snprintf(path,sizeof(path),"%s%s%d.dat",prefix,name,k);
  fp = fopen(path,"wb");
  if (fp == NULL) return 0;
  for (j = 0; j < f->ny; j ++)
    for (i = 0; i < f->nx; i ++)
      fwrite(&f->a[i+g][j+g],sizeof(double),1,fp);
  fclose(fp);
  return 1;
}

int main (int argc, char ** argv)
{
  static pawsim_context ctx;
  uint n,k,nsteps;
  double t0,t1,tsetup;

  if (argc < 3)
  {
    fprintf(stderr,"usage: ref_harness <param_file> <nsteps> [state_out_prefix]\n");
    return 1;
  }
  nsteps = (uint) strtoul(argv[2],NULL,10);
  memset(&ctx,0,sizeof(ctx));
  ctx.infname = argv[1];
  ctx.outdir = ".";
  t0 = now();
  pawsim_config_defaults(&ctx.cfg);
  if (!pawsim_config_read(ctx.infname,&ctx.cfg,stderr) || !pawsim_config_validate(&ctx.cfg,stderr))
    return 1;
  if (ctx.cfg.Lx <= 0) ctx.cfg.Lx = ctx.cfg.Ly * ctx.cfg.Nx / ctx.cfg.Ny;
  ctx.dx = ctx.cfg.Lx / ctx.cfg.Nx;
  ctx.dy = ctx.cfg.Ly / ctx.cfg.Ny;
  if (ctx.cfg.tmin < 0) ctx.cfg.tmin = 0;
  if (ctx.cfg.dt <= 0) { fprintf(stderr,"the harness needs dt\n"); return 1; }
  ctx.t = ctx.cfg.tmin;
  if (!pawsim_domain_init(&ctx.dom,ctx.cfg.Nx,ctx.cfg.Ny,3,!ctx.cfg.useWallEW,!ctx.cfg.useWallNS,0,0))
    return 1;
  if (!pawsim_state_alloc(&ctx.state,&ctx.cfg,&ctx.dom)
   || !pawsim_state_alloc(&ctx.tendency,&ctx.cfg,&ctx.dom)
   || !pawsim_state_alloc(&ctx.tendency_1,&ctx.cfg,&ctx.dom)
   || !pawsim_state_alloc(&ctx.tendency_2,&ctx.cfg,&ctx.dom)
   || !pawsim_work_alloc(&ctx.work,&ctx.cfg,&ctx.dom)
   || !pawsim_field2d_alloc(&ctx.pi,ctx.dom.nx,ctx.dom.ny,ctx.dom.nghost)
   || !pawsim_field2d_alloc(&ctx.pi_rhs,ctx.dom.nx,ctx.dom.ny,ctx.dom.nghost))
    return 1;
  pawsim_state_zero_prognostic(&ctx.tendency);
  pawsim_state_zero_prognostic(&ctx.tendency_1);
  pawsim_state_zero_prognostic(&ctx.tendency_2);
  pawsim_work_zero(&ctx.work);
  if (!pawsim_state_init(&ctx.state,&ctx.cfg,&ctx.dom,stderr)) return 1;
  pawsim_tendency_prepare_work_arrays(&ctx);
  pawsim_forcing_update(&ctx,ctx.t);
  pawsim_tendency_compute_deterministic_core(&ctx,&ctx.state);
  if (ctx.cfg.useRL)
  {
    uint it = pawsim_pressure_correct_rigid_lid(&ctx,false);
    printf("{\"phase\": \"prelim\", \"iters\": %u}\n",it);
    pawsim_tendency_prepare_work_arrays(&ctx);
    pawsim_forcing_update(&ctx,ctx.t);
    pawsim_tendency_compute_deterministic_core(&ctx,&ctx.state);
  }
  tsetup = now() - t0;
  printf("{\"phase\": \"setup\", \"seconds\": %.6f}\n",tsetup);
  fflush(stdout);
  for (n = 1; n <= nsteps; n ++)
  {
    uint it = 0;
    double tp;
    t0 = now();
    if (!pawsim_integrator_step(&ctx,n)) return 1;
    tp = now();
    if (ctx.cfg.useRL) it = pawsim_pressure_correct_rigid_lid(&ctx,true);
    t1 = now();
    printf("{\"phase\": \"step\", \"n\": %u, \"seconds\": %.6f, \"tendency_seconds\": %.6f, "
           "\"pressure_seconds\": %.6f, \"iters\": %u}\n",n,t1-t0,tp-t0,t1-tp,it);
    fflush(stdout);
  }
  if (argc > 3)
  {
    for (k = 0; k < ctx.cfg.Nlay; k ++)
    {
      if (!dump(argv[3],"U",k,&ctx.state.u[k]) || !dump(argv[3],"V",k,&ctx.state.v[k])
       || !dump(argv[3],"H",k,&ctx.state.h[k]))
        return 1;
    }
    if (!dump(argv[3],"P",0,&ctx.pi)) return 1;
  }
  return 0;
}
