/*
 * pawsim_oracle.c -- serial CPU restatement of PAWSIM's hot path (test infrastructure).
 *
 * See pawsim_oracle.h for scope. Layout: ghosted fields of width G = 3
 * (model_code/pawsim.c:28), x-fastest: A(f,i,j) = f->d[j*sx + i], with i, j in ghosted
 * coordinates; the owned cells are [G, G+nx) x [G, G+ny). Every floating-point
 * expression keeps the reference's association order, and the file is compiled with
 * -ffp-contract=off, so results match the reference's gcc -O3 x86-64 build bit for bit.
 */
#include "pawsim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define G 3
#define SQ(x) ((x)*(x))

typedef struct F2
{
  int nx, ny, sx, sy;
  double * d;
} F2;

#define A(f,i,j) ((f)->d[(size_t) (j)*(f)->sx + (size_t) (i)])

enum { K_SCALAR, K_Q, K_U, K_V };

typedef struct mg_level
{
  int Nx, Ny;
  double dx, dy;
  int power2;               /* transfer from this level to the next coarser is 2:1 */
  double *pi, *pi_temp, *rhs, *Hc, *Hw, *Hs, *Ow, *Os, *Osum, *rOsum;
  double *wmm, *wmp, *wpm, *wpp;
  int own_pi;
} mg_level;

struct orc_model
{
  orc_cfg c;
  int L, Nx, Ny;
  double dx, dy, t;
  /* state and three tendency levels (newest first) */
  F2 *u, *v, *h;
  F2 *tu[3], *tv[3], *th[3];
  /* static inputs */
  F2 hhs, hhb, omz, uLid, vLid, fbx, fby, hTime;
  F2 *taux, *tauy, *uRelax, *vRelax, *hRelax, *eRelax, *uTime, *vTime, *eTime;
  F2 *wdia_ff, *nu_u, *nu_v;
  double *gg, *geff;
  /* work arrays (work.h:93-193) */
  F2 *uw, *vw, *hw, *dtu, *dtv, *dth, *hwest, *hsouth, *hFsw, *hFss, *hFbw, *hFbs;
  F2 *hhq, *zeta, *qq, *al, *be, *ga, *de, *ep, *ph, *la, *mu, *pp, *KE, *MM;
  F2 *eta, *wdia, *wdiau, *wdiav, *Fdu, *Fdv, *gprime, *huu, *hvv;
  F2 hhsw, hhbw, hhs_west, hhs_south, hhb_west, hhb_south, Hc, Hw, Hs;
  F2 tauxw, tauyw, usqs, vsqs, uabss, usqb, vsqb, uabsb;
  F2 DDT, DDS, DD4T, DD4S, A2h, A2q, A4h, A4q, UU4, VV4, d2hx, d2hy, dhdx, dhdy;
  F2 pi, rhs;
  /* serial multigrid hierarchy (multigrid.c:20-63), index Ngrids-1 is finest */
  int mg_ready, Ngrids;
  mg_level * mg;
  double * Fmg;
  orc_pstats last;
};

/* ---------------------------------------------------------------- fields */

static int f2_alloc (F2 * f, int nx, int ny)
{
  f->nx = nx; f->ny = ny; f->sx = nx + 2*G; f->sy = ny + 2*G;
  f->d = (double *) calloc((size_t) f->sx*f->sy,sizeof(double));
  return f->d != NULL;
}

static F2 * f2_alloc_n (int n, int nx, int ny)
{
  F2 * a = (F2 *) calloc((size_t) n,sizeof(F2));
  int k;
  if (a == NULL) return NULL;
  for (k = 0; k < n; k ++)
  {
    if (!f2_alloc(&a[k],nx,ny)) return NULL;
  }
  return a;
}

static void f2_zero (F2 * f)
{
  memset(f->d,0,(size_t) f->sx*f->sy*sizeof(double));
}

static void f2_free_n (F2 * a, int n)
{
  int k;
  if (a == NULL) return;
  for (k = 0; k < n; k ++) free(a[k].d);
  free(a);
}

static void f2_fill (F2 * f, double v)
{
  size_t n = (size_t) f->sx*f->sy, p;
  for (p = 0; p < n; p ++) f->d[p] = v;
}

static void copy_owned (F2 * dst, const F2 * src)
{
  int i,j;
  for (j = G; j < G+dst->ny; j ++)
    for (i = G; i < G+dst->nx; i ++)
      A(dst,i,j) = A(src,i,j);
}

/* ----------------------------------------------------------- halo fills */

/* periodic copies (field.c:121-150): y over owned columns, x over every row */
static void per_y (F2 * f)
{
  int i,j;
  for (i = G; i < G+f->nx; i ++)
    for (j = 0; j < G; j ++)
    {
      A(f,i,j) = A(f,i,f->ny+j);
      A(f,i,G+f->ny+j) = A(f,i,G+j);
    }
}

static void per_x (F2 * f)
{
  int i,j;
  for (j = 0; j < f->sy; j ++)
    for (i = 0; i < G; i ++)
    {
      A(f,i,j) = A(f,f->nx+i,j);
      A(f,G+f->nx+i,j) = A(f,G+i,j);
    }
}

/* y-wall ghosts (field.c:158-198): owned columns, or every column for q fields */
static void wall_y (F2 * f, int kind)
{
  int i,j;
  int i0 = (kind == K_Q) ? 0 : G;
  int i1 = (kind == K_Q) ? f->sx : G+f->nx;
  for (i = i0; i < i1; i ++)
  {
    if (kind == K_V)
    {
      A(f,i,G) = 0;
      A(f,i,G+f->ny) = 0;
    }
    for (j = 0; j < G; j ++)
    {
      if (kind == K_Q)
      {
        A(f,i,j) = A(f,i,G);
        A(f,i,G+f->ny+j) = A(f,i,G+f->ny);
      }
      else if (kind == K_V)
      {
        A(f,i,j) = -A(f,i,2*G-j);
        A(f,i,G+f->ny+j) = -A(f,i,G+f->ny-j);
      }
      else
      {
        A(f,i,j) = A(f,i,2*G-j-1);
        A(f,i,G+f->ny+j) = A(f,i,G+f->ny-j-1);
      }
    }
  }
}

/* x-wall ghosts (field.c:204-241): every row */
static void wall_x (F2 * f, int kind)
{
  int i,j;
  for (j = 0; j < f->sy; j ++)
  {
    if (kind == K_U)
    {
      A(f,G,j) = 0;
      A(f,G+f->nx,j) = 0;
    }
    for (i = 0; i < G; i ++)
    {
      if (kind == K_Q)
      {
        A(f,i,j) = A(f,G,j);
        A(f,G+f->nx+i,j) = A(f,G+f->nx,j);
      }
      else if (kind == K_U)
      {
        A(f,i,j) = -A(f,2*G-i,j);
        A(f,G+f->nx+i,j) = -A(f,G+f->nx-i,j);
      }
      else
      {
        A(f,i,j) = A(f,2*G-i-1,j);
        A(f,G+f->nx+i,j) = A(f,G+f->nx-i-1,j);
      }
    }
  }
}

/* periodic-only refresh (field.c:353-427, serial branch) */
static void xch_internal (orc_model * m, F2 * f)
{
  if (!m->c.wall_ns) per_y(f);
  if (!m->c.wall_ew) per_x(f);
}

/*
 * Full refresh (field.c:458-532, serial branch). q fields keep the reference order. For
 * the other kinds the y direction is completed before the x direction, which equals the
 * reference except for its stale corners on x-periodic, y-walled domains.
 */
static void xch (orc_model * m, F2 * f, int kind)
{
  if (kind == K_Q)
  {
    if (!m->c.wall_ns) per_y(f);
    if (!m->c.wall_ew) per_x(f);
    if (m->c.wall_ns) wall_y(f,kind);
    if (m->c.wall_ew) wall_x(f,kind);
    return;
  }
  if (m->c.serial_corners)
  {
    /* serial order: periodic copies of every row or column first, then the wall ghosts */
    if (!m->c.wall_ns) per_y(f);
    if (!m->c.wall_ew) per_x(f);
    if (m->c.wall_ns) wall_y(f,kind);
    if (m->c.wall_ew) wall_x(f,kind);
    return;
  }
  if (m->c.wall_ns) wall_y(f,kind); else per_y(f);
  if (m->c.wall_ew) wall_x(f,kind); else per_x(f);
}

/* ------------------------------------------------------------ geometry */

/* centered face averages, the velocity-free branch of work.c:566-599 */
static void face_centered (const F2 * hh, F2 * hwst, F2 * hsth)
{
  int i,j;
  for (i = 1; i < hh->sx-1; i ++)
    for (j = 1; j < hh->sy-1; j ++)
    {
      A(hwst,i,j) = 0.5 * (A(hh,i,j)+A(hh,i-1,j));
      A(hsth,i,j) = 0.5 * (A(hh,i,j)+A(hh,i,j-1));
    }
}

static double minmod3 (double a, double b, double c)
{
  /* defs.c:1000-1014: zero unless all three share a sign, else the smallest magnitude */
  if ((a > 0) && (b > 0) && (c > 0)) return fmin(a,fmin(b,c));
  if ((a < 0) && (b < 0) && (c < 0)) return fmax(a,fmax(b,c));
  return 0;
}

/* velocity-dependent face thickness of one layer (work.c:566-684) */
static void face_layer (orc_model * m, F2 * hh, F2 * hwst, F2 * hsth, F2 * uu, F2 * vv)
{
  int i,j;
  int sch = m->c.thick_scheme;
  if (sch == 0)
  {
    face_centered(hh,hwst,hsth);
  }
  if (sch == 1)
  {
    for (i = 1; i < hh->sx-1; i ++)
      for (j = 1; j < hh->sy-1; j ++)
      {
        A(hsth,i,j) = (1.0/3) * ( A(hh,i,j)+A(hh,i,j-1)
                     + 0.25 * (A(hh,i+1,j)+A(hh,i-1,j)+A(hh,i+1,j-1)+A(hh,i-1,j-1)) );
        A(hwst,i,j) = (1.0/3) * ( A(hh,i,j)+A(hh,i-1,j)
                     + 0.25 * (A(hh,i,j+1)+A(hh,i-1,j+1)+A(hh,i,j-1)+A(hh,i-1,j-1)) );
      }
  }
  if (sch == 2)
  {
    for (i = 1; i < hh->sx-1; i ++)
      for (j = 1; j < hh->sy-1; j ++)
      {
        A(&m->d2hx,i,j) = A(hh,i+1,j) - 2*A(hh,i,j) + A(hh,i-1,j);
        A(&m->d2hy,i,j) = A(hh,i,j+1) - 2*A(hh,i,j) + A(hh,i,j-1);
      }
    for (i = 1; i < hh->sx-1; i ++)
      for (j = 1; j < hh->sy-1; j ++)
      {
        A(hsth,i,j) = 0.5 * (A(hh,i,j)+A(hh,i,j-1));
        A(hsth,i,j) -= (1/6.0) * ((A(vv,i,j) > 0) ? A(&m->d2hy,i,j-1) : A(&m->d2hy,i,j));
        A(hwst,i,j) = 0.5 * (A(hh,i,j)+A(hh,i-1,j));
        A(hwst,i,j) -= (1/6.0) * ((A(uu,i,j) > 0) ? A(&m->d2hx,i-1,j) : A(&m->d2hx,i,j));
      }
  }
  if (sch == 3)
  {
    double s = m->c.KT00_sigma;
    for (i = 1; i < hh->sx-1; i ++)
      for (j = 1; j < hh->sy-1; j ++)
      {
        A(&m->dhdx,i,j) = minmod3(s * (A(hh,i+1,j)-A(hh,i,j)),
                                  0.5 * (A(hh,i+1,j)-A(hh,i-1,j)),
                                  s * (A(hh,i,j)-A(hh,i-1,j)));
        A(&m->dhdy,i,j) = minmod3(s * (A(hh,i,j+1)-A(hh,i,j)),
                                  0.5 * (A(hh,i,j+1)-A(hh,i,j-1)),
                                  s * (A(hh,i,j)-A(hh,i,j-1)));
      }
    for (i = 1; i < hh->sx-1; i ++)
      for (j = 1; j < hh->sy-1; j ++)
      {
        double xm = A(hh,i-1,j) + 0.5*A(&m->dhdx,i-1,j);
        double xp = A(hh,i,j) - 0.5*A(&m->dhdx,i,j);
        double ym = A(hh,i,j-1) + 0.5*A(&m->dhdy,i,j-1);
        double yp = A(hh,i,j) + 0.5*A(&m->dhdy,i,j);
        A(hwst,i,j) = (A(uu,i,j) > 0) ? xm : xp;
        A(hsth,i,j) = (A(vv,i,j) > 0) ? ym : yp;
      }
  }
}

/* work.c:1124-1167 */
static void static_geometry (orc_model * m)
{
  int i,j;
  copy_owned(&m->hhsw,&m->hhs);
  copy_owned(&m->hhbw,&m->hhb);
  xch(m,&m->hhsw,K_SCALAR);
  xch(m,&m->hhbw,K_SCALAR);
  face_centered(&m->hhsw,&m->hhs_west,&m->hhs_south);
  face_centered(&m->hhbw,&m->hhb_west,&m->hhb_south);
  xch(m,&m->hhs_west,K_SCALAR);
  xch(m,&m->hhs_south,K_SCALAR);
  xch(m,&m->hhb_west,K_SCALAR);
  xch(m,&m->hhb_south,K_SCALAR);
  for (j = G; j < G+m->Ny; j ++)
    for (i = G; i < G+m->Nx; i ++)
      A(&m->Hc,i,j) = A(&m->hhs,i,j) - A(&m->hhb,i,j);
  xch(m,&m->Hc,K_SCALAR);
  face_centered(&m->Hc,&m->Hw,&m->Hs);
  xch(m,&m->Hw,K_SCALAR);
  xch(m,&m->Hs,K_SCALAR);
}

/* work.c:538-559 */
static void load_state (orc_model * m)
{
  int k;
  for (k = 0; k < m->L; k ++)
  {
    copy_owned(&m->uw[k],&m->u[k]);
    copy_owned(&m->vw[k],&m->v[k]);
    copy_owned(&m->hw[k],&m->h[k]);
    xch(m,&m->uw[k],K_U);
    xch(m,&m->vw[k],K_V);
    xch(m,&m->hw[k],K_SCALAR);
  }
}

static void state_halos (orc_model * m, F2 * u, F2 * v, F2 * h)
{
  int k;
  for (k = 0; k < m->L; k ++)
  {
    xch(m,&u[k],K_U);
    xch(m,&v[k],K_V);
    xch(m,&h[k],K_SCALAR);
  }
}

/* ------------------------------------------------------- tendency stages */

static void calc_face_thickness (orc_model * m)
{
  int k;
  for (k = 0; k < m->L; k ++)
  {
    face_layer(m,&m->hw[k],&m->hwest[k],&m->hsouth[k],&m->uw[k],&m->vw[k]);
    xch(m,&m->hwest[k],K_SCALAR);
    xch(m,&m->hsouth[k],K_SCALAR);
  }
}

/* work.c:1173-1203 */
static void calc_eta (orc_model * m)
{
  int k,i,j;
  for (k = m->L; k >= 0; k --)
  {
    for (j = 0; j < m->hhbw.sy; j ++)
      for (i = 0; i < m->hhbw.sx; i ++)
        A(&m->eta[k],i,j) = (k == m->L) ? A(&m->hhbw,i,j)
                                        : A(&m->eta[k+1],i,j) + A(&m->hw[k],i,j);
    xch(m,&m->eta[k],K_SCALAR);
  }
}

/* restoring.c:29-166 */
static void calc_wdia (orc_model * m)
{
  int k,i,j,L = m->L;
  for (k = 0; k < L+1; k ++) f2_zero(&m->wdia[k]);
  if (!m->c.use_wdia) return;
  if (m->c.use_wdia_file)
  {
    int n0 = 0, n1 = 0;
    double w0 = 1, w1 = 0;
    if ((m->c.wdia_nrecs > 1) && (m->c.wdia_period > 0))
    {
      double nflt = (fmod(m->t,m->c.wdia_period) / m->c.wdia_period) * m->c.wdia_nrecs;
      unsigned nm1 = (unsigned) floor(nflt), np1 = (unsigned) ceil(nflt);
      if (np1 == nm1) np1 = nm1 + 1;
      n0 = (int) nm1;
      n1 = (int) (np1 % (unsigned) m->c.wdia_nrecs);
      w0 = np1 - nflt;
      w1 = nflt - nm1;
    }
    for (k = 0; k < L+1; k ++)
    {
      F2 * a = &m->wdia_ff[n0*(L+1)+k];
      F2 * b = &m->wdia_ff[n1*(L+1)+k];
      for (j = G; j < G+m->Ny; j ++)
        for (i = G; i < G+m->Nx; i ++)
          A(&m->wdia[k],i,j) = w0*A(a,i,j) + w1*A(b,i,j);
    }
  }
  if (!m->c.use_relax)
  {
    for (k = 0; k < L+1; k ++) xch(m,&m->wdia[k],K_SCALAR);
  }
  if (m->c.use_relax)
  {
    for (j = G; j < G+m->Ny; j ++)
      for (i = G; i < G+m->Nx; i ++)
      {
        double acc = 0;
        for (k = L-1; k >= 0; k --)
        {
          if (A(&m->hTime,i,j) > 0)
          {
            acc += (A(&m->hw[k],i,j) - A(&m->hRelax[k],i,j)) / A(&m->hTime,i,j);
            A(&m->wdia[k],i,j) += acc;
          }
          if (A(&m->eTime[k],i,j) > 0)
          {
            A(&m->wdia[k],i,j) += (A(&m->eta[k],i,j) - A(&m->eRelax[k],i,j))
                                / A(&m->eTime[k],i,j);
          }
        }
      }
  }
  for (k = 0; k < L+1; k ++) xch(m,&m->wdia[k],K_SCALAR);
  for (k = 0; k < L+1; k ++)
  {
    for (j = G; j < G+m->Ny; j ++)
      for (i = G; i < G+m->Nx; i ++)
      {
        A(&m->wdiau[k],i,j) = 0.5*(A(&m->wdia[k],i,j) + A(&m->wdia[k],i-1,j));
        A(&m->wdiav[k],i,j) = 0.5*(A(&m->wdia[k],i,j) + A(&m->wdia[k],i,j-1));
      }
    xch(m,&m->wdiau[k],K_U);
    xch(m,&m->wdiav[k],K_V);
  }
}

/* diapycnal.c:27-66 (no tracer: g' is the layer reduced gravity) */
static void calc_gprime (orc_model * m)
{
  int k,i,j;
  for (k = 0; k < m->L; k ++) f2_zero(&m->gprime[k]);
  if ((m->c.conv_diff == 0) || (m->L < 2)) return;
  for (k = 1; k < m->L; k ++)
  {
    for (j = G; j < G+m->Ny; j ++)
      for (i = G; i < G+m->Nx; i ++)
        A(&m->gprime[k],i,j) = m->gg[k];
    xch(m,&m->gprime[k],K_SCALAR);
  }
}

/* work.c:1231-1288 */
static void calc_pv (orc_model * m)
{
  int k,i,j;
  for (k = 0; k < m->L; k ++)
  {
    F2 *u = &m->uw[k], *v = &m->vw[k], *h = &m->hw[k];
    int imax = h->sx - 2, jmax = h->sy - 2;
    f2_zero(&m->zeta[k]);
    f2_zero(&m->hhq[k]);
    f2_zero(&m->qq[k]);
    for (i = 1; i <= imax; i ++)
      for (j = 1; j <= jmax; j ++)
      {
        double z = (A(u,i,j-1)-A(u,i,j)) / m->dy + (A(v,i,j)-A(v,i-1,j)) / m->dx;
        double hq = 0.25 * (A(h,i,j) + A(h,i-1,j-1) + A(h,i-1,j) + A(h,i,j-1));
        A(&m->zeta[k],i,j) = z;
        A(&m->hhq[k],i,j) = hq;
        A(&m->qq[k],i,j) = (2*A(&m->omz,i,j) + z) / hq;
      }
    xch_internal(m,&m->zeta[k]);
    xch_internal(m,&m->hhq[k]);
    xch_internal(m,&m->qq[k]);
  }
}

/* work.c:1294-1404 */
static void calc_pv_coefficients (orc_model * m)
{
  int k,i,j,s = m->c.mom_scheme;
  for (k = 0; k < m->L; k ++)
  {
    F2 * q = &m->qq[k];
    f2_zero(&m->al[k]); f2_zero(&m->be[k]); f2_zero(&m->ga[k]); f2_zero(&m->de[k]);
    f2_zero(&m->ep[k]); f2_zero(&m->ph[k]); f2_zero(&m->la[k]); f2_zero(&m->mu[k]);
    for (i = 1; i < q->sx-1; i ++)
      for (j = 1; j < q->sy-1; j ++)
      {
        if ((s == 0) || (s == 1))
        {
          A(&m->al[k],i,j) = (2*A(q,i+1,j+1) + A(q,i,j+1) + 2*A(q,i,j) + A(q,i+1,j)) / 24;
          A(&m->be[k],i,j) = (A(q,i,j+1) + 2*A(q,i-1,j+1) + A(q,i-1,j) + 2*A(q,i,j)) / 24;
          A(&m->ga[k],i,j) = (2*A(q,i,j+1) + A(q,i-1,j+1) + 2*A(q,i-1,j) + A(q,i,j)) / 24;
          A(&m->de[k],i,j) = (A(q,i+1,j+1) + 2*A(q,i,j+1) + A(q,i,j) + 2*A(q,i+1,j)) / 24;
          A(&m->ep[k],i,j) = (A(q,i+1,j+1) + A(q,i,j+1) - A(q,i,j) - A(q,i+1,j)) / 24;
          A(&m->ph[k],i,j) = (-A(q,i+1,j+1) + A(q,i,j+1) + A(q,i,j) - A(q,i+1,j)) / 24;
        }
        else if ((s == 3) && (j < q->sy-2))
        {
          A(&m->al[k],i,j) = (2*A(q,i+1,j+1) + 3*A(q,i,j+1) + 2*A(q,i,j) + A(q,i+1,j)
                             - A(q,i,j+2) - A(q,i-1,j+1)) / 24;
          A(&m->be[k],i,j) = (3*A(q,i,j+1) + 2*A(q,i-1,j+1) + A(q,i-1,j) + 2*A(q,i,j)
                             - A(q,i+1,j+1) - A(q,i,j+2)) / 24;
          A(&m->ga[k],i,j) = (2*A(q,i,j+1) + A(q,i-1,j+1) + 2*A(q,i-1,j) + 3*A(q,i,j)
                             - A(q,i,j-1) - A(q,i+1,j)) / 24;
          A(&m->de[k],i,j) = (A(q,i+1,j+1) + 2*A(q,i,j+1) + 3*A(q,i,j) + 2*A(q,i+1,j)
                             - A(q,i-1,j) - A(q,i,j-1)) / 24;
          A(&m->ep[k],i,j) = (A(q,i+1,j+1) + A(q,i,j+1) - A(q,i,j) - A(q,i+1,j)) / 24;
          A(&m->ph[k],i,j) = (-A(q,i+1,j+1) + A(q,i,j+1) + A(q,i,j) - A(q,i+1,j)) / 24;
          A(&m->la[k],i,j) = (A(q,i+1,j) - A(q,i-1,j)) / 24;
          A(&m->mu[k],i,j) = (A(q,i,j-1) - A(q,i,j+1)) / 24;
        }
      }
    xch_internal(m,&m->al[k]); xch_internal(m,&m->be[k]);
    xch_internal(m,&m->ga[k]); xch_internal(m,&m->de[k]);
    xch_internal(m,&m->ep[k]); xch_internal(m,&m->ph[k]);
    xch_internal(m,&m->la[k]); xch_internal(m,&m->mu[k]);
  }
}

/* work.c:1410-1512 (no tracer) */
static void calc_bernoulli (orc_model * m)
{
  int k,i,j,s = m->c.mom_scheme;
  for (k = 0; k < m->L; k ++)
  {
    F2 *u = &m->uw[k], *v = &m->vw[k], *h = &m->hw[k];
    f2_zero(&m->pp[k]);
    f2_zero(&m->KE[k]);
    f2_zero(&m->MM[k]);
    for (i = 1; i < h->sx-1; i ++)
      for (j = 1; j < h->sy-1; j ++)
      {
        if (k == 0)
          A(&m->pp[k],i,j) = m->c.use_rl ? 0 : m->gg[0] * A(&m->eta[0],i,j);
        else
          A(&m->pp[k],i,j) = A(&m->pp[k-1],i,j) + m->gg[k] * A(&m->eta[k],i,j);

        if (s == 1)
        {
          A(&m->KE[k],i,j) =
            ( SQ(A(u,i+1,j)) + SQ(A(u,i,j))
            + 0.25 * ( SQ(A(u,i+1,j+1)) + SQ(A(u,i,j+1)) + SQ(A(u,i+1,j-1)) + SQ(A(u,i,j-1)) )
            + SQ(A(v,i,j+1)) + SQ(A(v,i,j))
            + 0.25 * ( SQ(A(v,i+1,j+1)) + SQ(A(v,i+1,j)) + SQ(A(v,i-1,j+1)) + SQ(A(v,i-1,j)) )
            ) / 6;
        }
        else if (s == 3)
        {
          if ((i < h->sx-2) && (j < h->sy-2))
          {
            A(&m->KE[k],i,j) =
              0.25 * ( (2.0/3.0)*SQ(A(u,i,j))
                     + (1.0/3.0)*SQ(0.5*(A(u,i-1,j)+A(u,i+1,j)))
                     + (2.0/3.0)*SQ(A(u,i+1,j))
                     + (1.0/3.0)*SQ(0.5*(A(u,i,j)+A(u,i+2,j)))
                     + (2.0/3.0)*SQ(A(v,i,j))
                     + (1.0/3.0)*SQ(0.5*(A(v,i,j-1)+A(v,i,j+1)))
                     + (2.0/3.0)*SQ(A(v,i,j+1))
                     + (1.0/3.0)*SQ(0.5*(A(v,i,j)+A(v,i,j+2))) );
          }
        }
        else
        {
          A(&m->KE[k],i,j) = ( SQ(A(u,i+1,j)) + SQ(A(u,i,j)) ) / 4
                           + ( SQ(A(v,i,j+1)) + SQ(A(v,i,j)) ) / 4;
        }

        A(&m->MM[k],i,j) = A(&m->pp[k],i,j);
        if (m->c.h0 != 0)
        {
          double h0 = m->c.h0, hc = A(h,i,j);
          A(&m->MM[k],i,j) -= m->geff[k] * (h0*h0*h0*h0) / (hc*hc*hc) / 3;
        }
      }
    xch(m,&m->pp[k],K_SCALAR);
    xch(m,&m->KE[k],K_SCALAR);
    xch(m,&m->MM[k],K_SCALAR);
  }
}

/* work.c:162-186 */
static void mass_fluxes (orc_model * m, int k)
{
  int i,j;
  f2_zero(&m->huu[k]);
  f2_zero(&m->hvv[k]);
  for (i = 1; i < m->hw[k].sx-1; i ++)
    for (j = 1; j < m->hw[k].sy-1; j ++)
    {
      A(&m->huu[k],i,j) = A(&m->uw[k],i,j) * A(&m->hwest[k],i,j);
      A(&m->hvv[k],i,j) = A(&m->vw[k],i,j) * A(&m->hsouth[k],i,j);
    }
  xch_internal(m,&m->huu[k]);
  xch_internal(m,&m->hvv[k]);
}

/* work.c:1520-1857 (budgets and active buoyancy omitted) */
static void calc_momentum (orc_model * m)
{
  int k,i,j;
  const orc_cfg * c = &m->c;
  double dx = m->dx, dy = m->dy;
  int useA2 = (c->A2 > 0) || (c->A2smag > 0);
  int useA4 = (c->A4 > 0) || (c->A4smag > 0);
  int useSmag = (c->A2smag > 0) || (c->A4smag > 0);
  double A2f = SQ(c->A2smag*fmax(dx,dy)/3.14159265358979323846);
  double mdx = fmax(dx,dy);
  double A4f = SQ(c->A4smag/3.14159265358979323846) * (mdx*mdx*mdx*mdx) / 8;
  double A4c = sqrt(c->A4);

  for (k = 0; k < m->L; k ++)
  {
    F2 *u = &m->uw[k], *v = &m->vw[k], *h = &m->hw[k];
    F2 *hq = &m->hhq[k], *hwst = &m->hwest[k], *hsth = &m->hsouth[k];
    F2 *huu = &m->huu[k], *hvv = &m->hvv[k];
    F2 *DT = &m->DDT, *DS = &m->DDS, *D4T = &m->DD4T, *D4S = &m->DD4S;
    f2_zero(&m->dtu[k]);
    f2_zero(&m->dtv[k]);
    mass_fluxes(m,k);

    if (useA2 || useA4)
    {
      f2_zero(DT); f2_zero(DS); f2_zero(&m->A2h); f2_zero(&m->A2q);
      f2_zero(&m->A4h); f2_zero(&m->A4q); f2_zero(&m->UU4); f2_zero(&m->VV4);
      f2_zero(D4T); f2_zero(D4S);
      for (i = 1; i < DT->sx-1; i ++)
        for (j = 1; j < DT->sy-1; j ++)
        {
          A(DT,i,j) = (A(u,i+1,j)-A(u,i,j))/dx - (A(v,i,j+1)-A(v,i,j))/dy;
          A(DS,i,j) = (A(u,i,j)-A(u,i,j-1))/dy + (A(v,i,j)-A(v,i-1,j))/dx;
        }
      if (useSmag)
      {
        for (i = 1; i < DT->sx-1; i ++)
          for (j = 1; j < DT->sy-1; j ++)
          {
            double DDq = sqrt(SQ(0.25*(A(DT,i,j)+A(DT,i-1,j)+A(DT,i,j-1)+A(DT,i-1,j-1)))
                            + SQ(A(DS,i,j)));
            double DDh = sqrt(SQ(A(DT,i,j))
                            + SQ(0.25*(A(DS,i,j)+A(DS,i+1,j)+A(DS,i,j+1)+A(DS,i+1,j+1))));
            A(&m->A2q,i,j) = fmax(c->A2,A2f*DDq);
            A(&m->A2h,i,j) = fmax(c->A2,A2f*DDh);
            A(&m->A4q,i,j) = sqrt(fmax(c->A4,A4f*DDq));
            A(&m->A4h,i,j) = sqrt(fmax(c->A4,A4f*DDh));
          }
      }
      else
      {
        for (i = 1; i < DT->sx-1; i ++)
          for (j = 1; j < DT->sy-1; j ++)
          {
            if (useA2) { A(&m->A2q,i,j) = c->A2; A(&m->A2h,i,j) = c->A2; }
            if (useA4) { A(&m->A4q,i,j) = A4c; A(&m->A4h,i,j) = A4c; }
          }
      }
      if (useA4)
      {
        F2 *Ah = &m->A4h, *Aq = &m->A4q, *U4 = &m->UU4, *V4 = &m->VV4;
        for (i = 1; i < U4->sx-1; i ++)
          for (j = 1; j < U4->sy-1; j ++)
          {
            A(U4,i,j) = (
                (A(Ah,i,j)*A(h,i,j)*A(DT,i,j) - A(Ah,i-1,j)*A(h,i-1,j)*A(DT,i-1,j)) / dx
              + (A(Aq,i,j+1)*A(hq,i,j+1)*A(DS,i,j+1) - A(Aq,i,j)*A(hq,i,j)*A(DS,i,j)) / dy
              ) / A(hwst,i,j);
            A(V4,i,j) = (
                (A(Aq,i+1,j)*A(hq,i+1,j)*A(DS,i+1,j) - A(Aq,i,j)*A(hq,i,j)*A(DS,i,j)) / dx
              - (A(Ah,i,j)*A(h,i,j)*A(DT,i,j) - A(Ah,i,j-1)*A(h,i,j-1)*A(DT,i,j-1)) / dy
              ) / A(hsth,i,j);
          }
        for (i = 1; i < D4T->sx-1; i ++)
          for (j = 1; j < D4T->sy-1; j ++)
          {
            A(D4T,i,j) = (A(U4,i+1,j)-A(U4,i,j))/dx - (A(V4,i,j+1)-A(V4,i,j))/dy;
            A(D4S,i,j) = (A(U4,i,j)-A(U4,i,j-1))/dy + (A(V4,i,j)-A(V4,i-1,j))/dx;
          }
      }
    }

    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        double hw_ = A(hwst,i,j), hs_ = A(hsth,i,j);
        double gM, gK, rq, a2 = 0, a4 = 0, ru, rv;
        F2 *al = &m->al[k], *be = &m->be[k], *ga = &m->ga[k], *de = &m->de[k];
        F2 *ep = &m->ep[k], *ph = &m->ph[k], *la = &m->la[k], *mu = &m->mu[k];
        F2 *q = &m->qq[k], *MM = &m->MM[k], *KE = &m->KE[k];

        gM = - (A(MM,i,j)-A(MM,i-1,j)) / dx;
        gK = - (A(KE,i,j)-A(KE,i-1,j)) / dx;
        rq = 0;
        if ((c->mom_scheme == 0) || (c->mom_scheme == 1))
        {
          rq += A(al,i,j)*A(hvv,i,j+1) + A(be,i,j)*A(hvv,i-1,j+1)
              + A(ga,i,j)*A(hvv,i-1,j) + A(de,i,j)*A(hvv,i,j)
              - A(ep,i,j)*A(huu,i+1,j) + A(ep,i-1,j)*A(huu,i-1,j);
        }
        else if (c->mom_scheme == 3)
        {
          rq += A(al,i,j)*A(hvv,i,j+1) + A(be,i,j)*A(hvv,i-1,j+1)
              + A(ga,i,j)*A(hvv,i-1,j) + A(de,i,j)*A(hvv,i,j)
              - A(ep,i,j)*A(huu,i+1,j) + A(ep,i-1,j)*A(huu,i-1,j)
              - A(la,i,j+1)*A(huu,i,j) + A(la,i,j)*A(huu,i,j-1);
        }
        else if (c->mom_scheme == 2)
        {
          rq += 0.25 * A(q,i,j) * (A(hvv,i,j) + A(hvv,i-1,j))
              + 0.25 * A(q,i,j+1) * (A(hvv,i,j+1) + A(hvv,i-1,j+1));
        }
        if (useA2)
        {
          a2 = ( (A(&m->A2h,i,j)*A(h,i,j)*A(DT,i,j) - A(&m->A2h,i-1,j)*A(h,i-1,j)*A(DT,i-1,j)) / dx
               + (A(&m->A2q,i,j+1)*A(hq,i,j+1)*A(DS,i,j+1) - A(&m->A2q,i,j)*A(hq,i,j)*A(DS,i,j)) / dy );
        }
        if (useA4)
        {
          a4 = -( (A(&m->A4h,i,j)*A(h,i,j)*A(D4T,i,j) - A(&m->A4h,i-1,j)*A(h,i-1,j)*A(D4T,i-1,j)) / dx
                + (A(&m->A4q,i,j+1)*A(hq,i,j+1)*A(D4S,i,j+1) - A(&m->A4q,i,j)*A(hq,i,j)*A(D4S,i,j)) / dy );
        }
        ru = gM + gK + rq + ((hw_ != 0) ? (a2+a4+0.0)/hw_ : 0);

        gM = - (A(MM,i,j)-A(MM,i,j-1)) / dy;
        gK = - (A(KE,i,j)-A(KE,i,j-1)) / dy;
        rq = 0;
        a2 = 0;
        a4 = 0;
        if ((c->mom_scheme == 0) || (c->mom_scheme == 1))
        {
          rq += A(ph,i,j-1)*A(hvv,i,j-1) - A(ph,i,j)*A(hvv,i,j+1)
              - A(ga,i+1,j)*A(huu,i+1,j) - A(de,i,j)*A(huu,i,j)
              - A(al,i,j-1)*A(huu,i,j-1) - A(be,i+1,j-1)*A(huu,i+1,j-1);
        }
        else if (c->mom_scheme == 3)
        {
          rq += A(ph,i,j-1)*A(hvv,i,j-1) - A(ph,i,j)*A(hvv,i,j+1)
              - A(ga,i+1,j)*A(huu,i+1,j) - A(de,i,j)*A(huu,i,j)
              - A(al,i,j-1)*A(huu,i,j-1) - A(be,i+1,j-1)*A(huu,i+1,j-1)
              - A(mu,i+1,j)*A(hvv,i,j) + A(mu,i,j)*A(hvv,i-1,j);
        }
        else if (c->mom_scheme == 2)
        {
          rq -= 0.25 * A(q,i,j) * (A(huu,i,j) + A(huu,i,j-1))
              + 0.25 * A(q,i+1,j) * (A(huu,i+1,j) + A(huu,i+1,j-1));
        }
        if (useA2)
        {
          a2 = ( (A(&m->A2q,i+1,j)*A(hq,i+1,j)*A(DS,i+1,j) - A(&m->A2q,i,j)*A(hq,i,j)*A(DS,i,j)) / dx
               - (A(&m->A2h,i,j)*A(h,i,j)*A(DT,i,j) - A(&m->A2h,i,j-1)*A(h,i,j-1)*A(DT,i,j-1)) / dy );
        }
        if (useA4)
        {
          a4 = -( (A(&m->A4q,i+1,j)*A(hq,i+1,j)*A(D4S,i+1,j) - A(&m->A4q,i,j)*A(hq,i,j)*A(D4S,i,j)) / dx
                - (A(&m->A4h,i,j)*A(h,i,j)*A(D4T,i,j) - A(&m->A4h,i,j-1)*A(h,i,j-1)*A(D4T,i,j-1)) / dy );
        }
        rv = gM + gK + rq + ((hs_ != 0) ? (a2+a4+0.0)/hs_ : 0);

        A(&m->dtu[k],i,j) = ru;
        A(&m->dtv[k],i,j) = rv;
      }
    xch(m,&m->dtu[k],K_U);
    xch(m,&m->dtv[k],K_V);
  }
}

/* diapycnal.c:72-133 */
static void diapycnal_fluxes (orc_model * m)
{
  int k,i,j;
  for (k = 0; k < m->L+1; k ++) { f2_zero(&m->Fdu[k]); f2_zero(&m->Fdv[k]); }
  if (!m->c.use_diavisc || (m->L < 2)) return;
  for (k = 1; k < m->L; k ++)
    for (j = G; j < G+m->Ny; j ++)
      for (i = G; i < G+m->Nx; i ++)
      {
        double dzu = 0.5*(A(&m->hwest[k],i,j) + A(&m->hwest[k-1],i,j));
        double dzv = 0.5*(A(&m->hsouth[k],i,j) + A(&m->hsouth[k-1],i,j));
        double nuu = A(&m->nu_u[k],i,j), nuv = A(&m->nu_v[k],i,j);
        if (m->c.conv_diff != 0)
        {
          if ((A(&m->gprime[k],i,j) < 0) || (A(&m->gprime[k],i-1,j) < 0)) nuu += m->c.conv_diff;
          if ((A(&m->gprime[k],i,j) < 0) || (A(&m->gprime[k],i,j-1) < 0)) nuv += m->c.conv_diff;
        }
        if (dzu != 0) A(&m->Fdu[k],i,j) = nuu * (A(&m->uw[k-1],i,j) - A(&m->uw[k],i,j)) / dzu;
        if (dzv != 0) A(&m->Fdv[k],i,j) = nuv * (A(&m->vw[k-1],i,j) - A(&m->vw[k],i,j)) / dzv;
      }
}

/* diapycnal.c:203-291 */
static void diapycnal_apply (orc_model * m)
{
  int k,i,j,L = m->L;
  calc_gprime(m);
  diapycnal_fluxes(m);
  if (!m->c.use_wdia && !m->c.use_diavisc) return;
  for (k = 0; k < L; k ++)
  {
    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        double hw_ = A(&m->hwest[k],i,j), hs_ = A(&m->hsouth[k],i,j);
        if (m->c.use_wdia)
        {
          double uc = A(&m->uw[k],i,j), vc = A(&m->vw[k],i,j);
          double up = (k == 0) ? 0 : A(&m->uw[k-1],i,j);
          double um = (k == L-1) ? 0 : A(&m->uw[k+1],i,j);
          double vp = (k == 0) ? 0 : A(&m->vw[k-1],i,j);
          double vm = (k == L-1) ? 0 : A(&m->vw[k+1],i,j);
          double wu0 = A(&m->wdiau[k],i,j), wu1 = A(&m->wdiau[k+1],i,j);
          double wv0 = A(&m->wdiav[k],i,j), wv1 = A(&m->wdiav[k+1],i,j);
          double dup = (wu0 > 0) ? 0 : up-uc;
          double dum = (wu1 > 0) ? uc-um : 0;
          double dvp = (wv0 > 0) ? 0 : vp-vc;
          double dvm = (wv1 > 0) ? vc-vm : 0;
          if (hw_ != 0) A(&m->dtu[k],i,j) += (- (wu0*dup + wu1*dum)) / hw_;
          if (hs_ != 0) A(&m->dtv[k],i,j) += (- (wv0*dvp + wv1*dvm)) / hs_;
        }
        if (m->c.use_diavisc)
        {
          if (hw_ != 0) A(&m->dtu[k],i,j) += (A(&m->Fdu[k],i,j) - A(&m->Fdu[k+1],i,j)) / hw_;
          if (hs_ != 0) A(&m->dtv[k],i,j) += (A(&m->Fdv[k],i,j) - A(&m->Fdv[k+1],i,j)) / hs_;
        }
      }
    xch(m,&m->dtu[k],K_U);
    xch(m,&m->dtv[k],K_V);
  }
}

/* forcing.c:30-89 */
static void forcing_update (orc_model * m, double t)
{
  int i,j,n0 = 0,n1 = 0;
  double w0 = 1, w1 = 0;
  f2_zero(&m->tauxw);
  f2_zero(&m->tauyw);
  if (!m->c.use_wind) return;
  if ((m->c.tau_nrecs > 1) && (m->c.tau_period > 0))
  {
    double nflt = (fmod(t,m->c.tau_period) / m->c.tau_period) * m->c.tau_nrecs;
    unsigned nm1 = (unsigned) floor(nflt), np1 = (unsigned) ceil(nflt);
    if (np1 == nm1) np1 = nm1 + 1;
    n0 = (int) nm1;
    n1 = (int) (np1 % (unsigned) m->c.tau_nrecs);
    w0 = np1 - nflt;
    w1 = nflt - nm1;
  }
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
    {
      A(&m->tauxw,i,j) = w0*A(&m->taux[n0],i,j) + w1*A(&m->taux[n1],i,j);
      A(&m->tauyw,i,j) = w0*A(&m->tauy[n0],i,j) + w1*A(&m->tauy[n1],i,j);
    }
  xch(m,&m->tauxw,K_SCALAR);
  xch(m,&m->tauyw,K_SCALAR);
}

/* work.c:2151-2241 */
static void surface_fraction (orc_model * m)
{
  int i,j,k,L = m->L;
  for (k = 0; k < L; k ++) { f2_zero(&m->hFsw[k]); f2_zero(&m->hFss[k]); }
  if (m->c.hsml <= 0)
  {
    f2_fill(&m->hFsw[0],1);
    f2_fill(&m->hFss[0],1);
  }
  else
  {
    for (i = 1; i < m->hFsw[0].sx-1; i ++)
      for (j = 1; j < m->hFsw[0].sy-1; j ++)
      {
        double zw = A(&m->hhs_west,i,j) - m->c.hsml;
        double zs = A(&m->hhs_south,i,j) - m->c.hsml;
        double ew = A(&m->hhs_west,i,j), es = A(&m->hhs_south,i,j);
        double sw = 0, ss = 0;
        for (k = 0; k < L; k ++)
        {
          double ewl = ew - A(&m->hwest[k],i,j);
          double esl = es - A(&m->hsouth[k],i,j);
          if (sw < 1.0)
          {
            double he;
            zw -= fmin(m->c.hmin_surf,A(&m->hwest[k],i,j));
            he = fmax(ew,zw) - fmax(ewl,zw);
            he = fmax(he-m->c.hmin_surf,0);
            A(&m->hFsw[k],i,j) = he / m->c.hsml;
            sw += A(&m->hFsw[k],i,j);
          }
          if (ss < 1.0)
          {
            double he;
            zs -= fmin(m->c.hmin_surf,A(&m->hsouth[k],i,j));
            he = fmax(es,zs) - fmax(esl,zs);
            he = fmax(he-m->c.hmin_surf,0);
            A(&m->hFss[k],i,j) = he / m->c.hsml;
            ss += A(&m->hFss[k],i,j);
          }
          ew = ewl;
          es = esl;
        }
      }
  }
  for (k = 0; k < L; k ++) { xch(m,&m->hFsw[k],K_U); xch(m,&m->hFss[k],K_V); }
}

/* work.c:2248-2340 */
static void bottom_fraction (orc_model * m)
{
  int i,j,k,L = m->L;
  for (k = 0; k < L; k ++) { f2_zero(&m->hFbw[k]); f2_zero(&m->hFbs[k]); }
  if (m->c.hbbl <= 0)
  {
    f2_fill(&m->hFbw[L-1],1);
    f2_fill(&m->hFbs[L-1],1);
  }
  else
  {
    for (i = 1; i < m->hFbw[0].sx-1; i ++)
      for (j = 1; j < m->hFbw[0].sy-1; j ++)
      {
        double zw = A(&m->hhb_west,i,j) + m->c.hbbl;
        double zs = A(&m->hhb_south,i,j) + m->c.hbbl;
        double ewl = A(&m->hhb_west,i,j), esl = A(&m->hhb_south,i,j);
        double sw = 0, ss = 0;
        for (k = L; k > 0; k --)
        {
          int kk = k - 1;
          double ewu = ewl + A(&m->hwest[kk],i,j);
          double esu = esl + A(&m->hsouth[kk],i,j);
          if (sw < 1.0)
          {
            double he;
            zw += fmin(m->c.hmin_bot,A(&m->hwest[kk],i,j));
            he = fmin(ewu,zw) - fmin(ewl,zw);
            he = fmax(he-m->c.hmin_bot,0);
            A(&m->hFbw[kk],i,j) = he / m->c.hbbl;
            sw += A(&m->hFbw[kk],i,j);
          }
          if (ss < 1.0)
          {
            double he;
            zs += fmin(m->c.hmin_bot,A(&m->hsouth[kk],i,j));
            he = fmin(esu,zs) - fmin(esl,zs);
            he = fmax(he-m->c.hmin_bot,0);
            A(&m->hFbs[kk],i,j) = he / m->c.hbbl;
            ss += A(&m->hFbs[kk],i,j);
          }
          ewl = ewu;
          esl = esu;
        }
      }
  }
  for (k = 0; k < L; k ++) { xch(m,&m->hFbw[k],K_U); xch(m,&m->hFbs[k],K_V); }
}

/* forcing.c:95-143 */
static void surface_drag_speed (orc_model * m)
{
  int i,j,k;
  double wfb = m->c.wind_feedback ? 0.3 : 0.0;
  for (i = 0; i < m->usqs.sx; i ++)
    for (j = 0; j < m->usqs.sy; j ++)
    {
      double us = 0, vs = 0, ur, vr;
      if (m->c.hsml > 0)
      {
        for (k = 0; k < m->L; k ++)
        {
          us += A(&m->uw[k],i,j) * A(&m->hFsw[k],i,j);
          vs += A(&m->vw[k],i,j) * A(&m->hFss[k],i,j);
        }
      }
      else
      {
        us = A(&m->uw[0],i,j);
        vs = A(&m->vw[0],i,j);
      }
      ur = (1.0-wfb)*us - A(&m->uLid,i,j);
      vr = (1.0-wfb)*vs - A(&m->vLid,i,j);
      A(&m->usqs,i,j) = ur * ur;
      A(&m->vsqs,i,j) = vr * vr;
    }
  for (i = 0; i < m->uabss.sx-1; i ++)
    for (j = 0; j < m->uabss.sy-1; j ++)
      A(&m->uabss,i,j) = sqrt(0.5*(A(&m->usqs,i,j)+A(&m->usqs,i+1,j))
                            + 0.5*(A(&m->vsqs,i,j)+A(&m->vsqs,i,j+1)));
}

/* forcing.c:149-395 */
static void forcing_apply (orc_model * m)
{
  int i,j,k,L = m->L;
  const orc_cfg * c = &m->c;
  int surf = (c->lin_drag_surf > 0) || (c->quad_drag_surf > 0);
  int bot = (c->lin_drag > 0) || (c->quad_drag > 0);
  double wfb = c->wind_feedback ? 0.3 : 0.0;

  if (c->use_wind || surf) surface_fraction(m);
  if (bot) bottom_fraction(m);
  if (c->quad_drag_surf > 0) surface_drag_speed(m);
  if (c->quad_drag > 0)
  {
    for (i = 0; i < m->usqb.sx; i ++)
      for (j = 0; j < m->usqb.sy; j ++)
      {
        double ub = 0, vb = 0;
        if (c->hbbl > 0)
        {
          for (k = 0; k < L; k ++)
          {
            ub += A(&m->uw[k],i,j) * A(&m->hFbw[k],i,j);
            vb += A(&m->vw[k],i,j) * A(&m->hFbs[k],i,j);
          }
        }
        else
        {
          ub = A(&m->uw[L-1],i,j);
          vb = A(&m->vw[L-1],i,j);
        }
        A(&m->usqb,i,j) = ub * ub;
        A(&m->vsqb,i,j) = vb * vb;
      }
    for (i = 0; i < m->uabsb.sx-1; i ++)
      for (j = 0; j < m->uabsb.sy-1; j ++)
        A(&m->uabsb,i,j) = sqrt(0.5*(A(&m->usqb,i,j)+A(&m->usqb,i+1,j))
                              + 0.5*(A(&m->vsqb,i,j)+A(&m->vsqb,i,j+1)));
  }
  if (!c->use_wind && !c->use_fbaro && !surf && !bot) return;

  for (k = 0; k < L; k ++)
  {
    F2 *du = &m->dtu[k], *dv = &m->dtv[k], *u = &m->uw[k], *v = &m->vw[k];
    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        double hw_ = A(&m->hwest[k],i,j), hs_ = A(&m->hsouth[k],i,j);
        if (c->use_wind)
        {
          double r = A(&m->tauxw,i,j) * A(&m->hFsw[k],i,j);
          if (hw_ != 0) A(du,i,j) += r / hw_;
          r = A(&m->tauyw,i,j) * A(&m->hFss[k],i,j);
          if (hs_ != 0) A(dv,i,j) += r / hs_;
        }
        if (c->use_fbaro)
        {
          A(du,i,j) += A(&m->fbx,i,j);
          A(dv,i,j) += A(&m->fby,i,j);
        }
        if ((c->lin_drag > 0) && (hw_ != 0))
          A(du,i,j) += (-c->lin_drag * A(u,i,j) * A(&m->hFbw[k],i,j)) / hw_;
        if ((c->lin_drag > 0) && (hs_ != 0))
          A(dv,i,j) += (-c->lin_drag * A(v,i,j) * A(&m->hFbs[k],i,j)) / hs_;
        if ((c->lin_drag_surf > 0) && (hw_ != 0))
        {
          double r = -c->lin_drag_surf * (A(u,i,j)-A(&m->uLid,i,j)) * A(&m->hFsw[k],i,j);
          if (!c->ocean_surf_drag && c->use_rl && (A(&m->hhs_west,i,j) >= 0)) r = 0;
          A(du,i,j) += r / hw_;
        }
        if ((c->lin_drag_surf > 0) && (hs_ != 0))
        {
          double r = -c->lin_drag_surf * (A(v,i,j)-A(&m->vLid,i,j)) * A(&m->hFss[k],i,j);
          if (!c->ocean_surf_drag && c->use_rl && (A(&m->hhs_south,i,j) >= 0)) r = 0;
          A(dv,i,j) += r / hs_;
        }
        if ((c->quad_drag > 0) && (hw_ != 0))
        {
          double ua = 0.5*(A(&m->uabsb,i,j)+A(&m->uabsb,i-1,j));
          A(du,i,j) -= c->quad_drag * ua * A(u,i,j) * A(&m->hFbw[k],i,j) / hw_;
        }
        if ((c->quad_drag > 0) && (hs_ != 0))
        {
          double ua = 0.5*(A(&m->uabsb,i,j)+A(&m->uabsb,i,j-1));
          A(dv,i,j) -= c->quad_drag * ua * A(v,i,j) * A(&m->hFbs[k],i,j) / hs_;
        }
        if ((c->quad_drag_surf > 0) && (hw_ != 0))
        {
          double ua = 0.5*(A(&m->uabss,i,j)+A(&m->uabss,i-1,j));
          double r = -c->quad_drag_surf * ua * ((1.0-wfb)*A(u,i,j)-A(&m->uLid,i,j))
                   * A(&m->hFsw[k],i,j);
          if (!c->ocean_surf_drag && c->use_rl && (A(&m->hhs_west,i,j) >= 0)) r = 0;
          A(du,i,j) += r / hw_;
        }
        if ((c->quad_drag_surf > 0) && (hs_ != 0))
        {
          double ua = 0.5*(A(&m->uabss,i,j)+A(&m->uabss,i,j-1));
          double r = -c->quad_drag_surf * ua * ((1.0-wfb)*A(v,i,j)-A(&m->vLid,i,j))
                   * A(&m->hFss[k],i,j);
          if (!c->ocean_surf_drag && c->use_rl && (A(&m->hhs_south,i,j) >= 0)) r = 0;
          A(dv,i,j) += r / hs_;
        }
      }
    xch(m,du,K_U);
    xch(m,dv,K_V);
  }
}

/* restoring.c:172-220 */
static void restoring_apply (orc_model * m)
{
  int i,j,k;
  if (!m->c.use_relax) return;
  for (k = 0; k < m->L; k ++)
  {
    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        if (A(&m->uTime[k],i,j) > 0)
          A(&m->dtu[k],i,j) += - (A(&m->uw[k],i,j) - A(&m->uRelax[k],i,j)) / A(&m->uTime[k],i,j);
        if (A(&m->vTime[k],i,j) > 0)
          A(&m->dtv[k],i,j) += - (A(&m->vw[k],i,j) - A(&m->vRelax[k],i,j)) / A(&m->vTime[k],i,j);
      }
    xch(m,&m->dtu[k],K_U);
    xch(m,&m->dtv[k],K_V);
  }
}

/* work.c:1864-1941 */
static void calc_thickness (orc_model * m)
{
  int k,i,j;
  for (k = 0; k < m->L; k ++)
  {
    f2_zero(&m->dth[k]);
    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        double adv = (A(&m->huu[k],i,j)-A(&m->huu[k],i+1,j)) / m->dx
                   + (A(&m->hvv[k],i,j)-A(&m->hvv[k],i,j+1)) / m->dy;
        double rel = - (A(&m->wdia[k],i,j) - A(&m->wdia[k+1],i,j));
        A(&m->dth[k],i,j) = adv + rel;
      }
    xch(m,&m->dth[k],K_SCALAR);
  }
}

/* tendency.c:49-75 */
static void core (orc_model * m)
{
  calc_face_thickness(m);
  calc_eta(m);
  calc_wdia(m);
  calc_gprime(m);
  calc_pv(m);
  calc_pv_coefficients(m);
  calc_bernoulli(m);
  calc_momentum(m);
  diapycnal_apply(m);
  forcing_apply(m);
  restoring_apply(m);
  calc_thickness(m);
}

void orc_prepare_and_core (orc_model * m)
{
  load_state(m);
  static_geometry(m);
  forcing_update(m,m->t);
  core(m);
}

/* tendency.c:81-115: the newest history level receives the owned tendency values */
int orc_tendency (orc_model * m)
{
  int k;
  forcing_update(m,m->t);
  for (k = 0; k < m->L; k ++)
  {
    f2_zero(&m->tu[0][k]); f2_zero(&m->tv[0][k]); f2_zero(&m->th[0][k]);
  }
  load_state(m);
  static_geometry(m);
  core(m);
  for (k = 0; k < m->L; k ++)
  {
    copy_owned(&m->tu[0][k],&m->dtu[k]);
    copy_owned(&m->tv[0][k],&m->dtv[k]);
    copy_owned(&m->th[0][k],&m->dth[k]);
  }
  state_halos(m,m->tu[0],m->tv[0],m->th[0]);
  return 0;
}

/* ----------------------------------------------------------- integrator */

static void ab1 (orc_model * m, F2 * s, F2 * f0)
{
  int i,j;
  double dt = m->c.dt;
  for (i = G; i < G+s->nx; i ++)
    for (j = G; j < G+s->ny; j ++)
      A(s,i,j) += dt * A(f0,i,j);
}

static void ab2 (orc_model * m, F2 * s, F2 * f0, F2 * f1)
{
  int i,j;
  double dt = m->c.dt;
  for (i = G; i < G+s->nx; i ++)
    for (j = G; j < G+s->ny; j ++)
      A(s,i,j) += (3*dt/2) * A(f0,i,j) - (dt/2) * A(f1,i,j);
}

static void ab3 (orc_model * m, F2 * s, F2 * f0, F2 * f1, F2 * f2)
{
  int i,j;
  double dt = m->c.dt;
  for (i = G; i < G+s->nx; i ++)
    for (j = G; j < G+s->ny; j ++)
      A(s,i,j) += (23*dt/12) * A(f0,i,j) - (4*dt/3) * A(f1,i,j) + (5*dt/12) * A(f2,i,j);
}

/* integrator.c:127-132 */
static void shift_history (orc_model * m)
{
  int k;
  for (k = 0; k < m->L; k ++)
  {
    copy_owned(&m->tu[2][k],&m->tu[1][k]); copy_owned(&m->tv[2][k],&m->tv[1][k]);
    copy_owned(&m->th[2][k],&m->th[1][k]);
    copy_owned(&m->tu[1][k],&m->tu[0][k]); copy_owned(&m->tv[1][k],&m->tv[0][k]);
    copy_owned(&m->th[1][k],&m->th[0][k]);
  }
}

/* integrator.c:138-198 */
int orc_integrator_step (orc_model * m, int n)
{
  int k,sch = m->c.ts_scheme;
  orc_tendency(m);
  for (k = 0; k < m->L; k ++)
  {
    F2 * s[3] = { &m->u[k], &m->v[k], &m->h[k] };
    F2 * f0[3] = { &m->tu[0][k], &m->tv[0][k], &m->th[0][k] };
    F2 * f1[3] = { &m->tu[1][k], &m->tv[1][k], &m->th[1][k] };
    F2 * f2[3] = { &m->tu[2][k], &m->tv[2][k], &m->th[2][k] };
    int v;
    for (v = 0; v < 3; v ++)
    {
      if ((sch == 3) || (n == 1)) ab1(m,s[v],f0[v]);
      else if ((sch == 4) || (n == 2)) ab2(m,s[v],f0[v],f1[v]);
      else ab3(m,s[v],f0[v],f1[v],f2[v]);
    }
  }
  if (!((sch == 5) && (n == 1))) shift_history(m);
  m->t += m->c.dt;
  state_halos(m,m->u,m->v,m->h);
  return 0;
}

/* ------------------------------------------------------------- pressure */

/* pressure.c:55-88: serial-order global sum, i outer and j inner */
static double owned_mean (orc_model * m, const F2 * f)
{
  int i,j;
  double s = 0;
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
      s += A(f,i,j);
  return s / ((double) m->Nx * (double) m->Ny);
}

static void subtract_mean (orc_model * m, F2 * f)
{
  int i,j;
  double mean = owned_mean(m,f);
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
      A(f,i,j) -= mean;
}

/* pressure.c:525-561 */
static void correct_thickness (orc_model * m)
{
  int i,j,k;
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
    {
      double tot = 0, err;
      for (k = 0; k < m->L; k ++) tot += A(&m->h[k],i,j);
      if (tot == 0) continue;
      err = tot - A(&m->Hc,i,j);
      for (k = 0; k < m->L; k ++) A(&m->h[k],i,j) *= (1 - err / tot);
    }
  state_halos(m,m->u,m->v,m->h);
}

/* work.c:865-1030 + 1037-1118: face thickness on the global field with wrapped indices */
static void face_thickness_global (orc_model * m)
{
  int Nx = m->Nx, Ny = m->Ny, k, i, j, sch = m->c.thick_scheme;
  double *d2x = NULL, *d2y = NULL;
#define GH(f,ii,jj) A(f,G+((ii)%Nx),G+((jj)%Ny))
  for (k = 0; k < m->L; k ++)
  {
    F2 *hh = &m->hw[k], *uu = &m->uw[k], *vv = &m->vw[k];
    F2 *hw_ = &m->hwest[k], *hs_ = &m->hsouth[k];
    f2_zero(hw_);
    f2_zero(hs_);
    if (sch == 0)
    {
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, jm1 = (j+Ny-1) % Ny;
          A(hw_,G+i,G+j) = 0.5*(GH(hh,i,j)+GH(hh,im1,j));
          A(hs_,G+i,G+j) = 0.5*(GH(hh,i,j)+GH(hh,i,jm1));
        }
    }
    else if (sch == 1)
    {
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, ip1 = (i+1) % Nx, jm1 = (j+Ny-1) % Ny, jp1 = (j+1) % Ny;
          if (m->c.wall_ew && (i == 0))
            A(hs_,G+i,G+j) = (1.0/3) * (1.25*(GH(hh,i,j)+GH(hh,i,jm1))
                                      + 0.25*(GH(hh,ip1,j)+GH(hh,ip1,jm1)));
          else if (m->c.wall_ew && (i == Nx-1))
            A(hs_,G+i,G+j) = (1.0/3) * (1.25*(GH(hh,i,j)+GH(hh,i,jm1))
                                      + 0.25*(GH(hh,im1,j)+GH(hh,im1,jm1)));
          else
            A(hs_,G+i,G+j) = (1.0/3) * (GH(hh,i,j)+GH(hh,i,jm1)
                                      + 0.25*(GH(hh,ip1,j)+GH(hh,im1,j)
                                             + GH(hh,ip1,jm1)+GH(hh,im1,jm1)));
          if (m->c.wall_ns && (j == 0))
            A(hw_,G+i,G+j) = (1.0/3) * (1.25*(GH(hh,i,j)+GH(hh,im1,j))
                                      + 0.25*(GH(hh,i,jp1)+GH(hh,im1,jp1)));
          else if (m->c.wall_ns && (j == Ny-1))
            A(hw_,G+i,G+j) = (1.0/3) * (1.25*(GH(hh,i,j)+GH(hh,im1,j))
                                      + 0.25*(GH(hh,i,jm1)+GH(hh,im1,jm1)));
          else
            A(hw_,G+i,G+j) = (1.0/3) * (GH(hh,i,j)+GH(hh,im1,j)
                                      + 0.25*(GH(hh,i,jp1)+GH(hh,im1,jp1)
                                             + GH(hh,i,jm1)+GH(hh,im1,jm1)));
        }
    }
    else if (sch == 2)
    {
      d2x = (double *) calloc((size_t) Nx*Ny,sizeof(double));
      d2y = (double *) calloc((size_t) Nx*Ny,sizeof(double));
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, ip1 = (i+1) % Nx, jm1 = (j+Ny-1) % Ny, jp1 = (j+1) % Ny;
          d2x[i*Ny+j] = GH(hh,ip1,j)-2*GH(hh,i,j)+GH(hh,im1,j);
          d2y[i*Ny+j] = GH(hh,i,jp1)-2*GH(hh,i,j)+GH(hh,i,jm1);
        }
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, jm1 = (j+Ny-1) % Ny;
          A(hs_,G+i,G+j) = 0.5*(GH(hh,i,j)+GH(hh,i,jm1))
                         - (1/6.0) * ((GH(vv,i,j) > 0) ? d2y[i*Ny+jm1] : d2y[i*Ny+j]);
          A(hw_,G+i,G+j) = 0.5*(GH(hh,i,j)+GH(hh,im1,j))
                         - (1/6.0) * ((GH(uu,i,j) > 0) ? d2x[im1*Ny+j] : d2x[i*Ny+j]);
        }
      free(d2x); free(d2y);
    }
    else
    {
      double s = m->c.KT00_sigma;
      d2x = (double *) calloc((size_t) Nx*Ny,sizeof(double));
      d2y = (double *) calloc((size_t) Nx*Ny,sizeof(double));
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, ip1 = (i+1) % Nx, jm1 = (j+Ny-1) % Ny, jp1 = (j+1) % Ny;
          d2x[i*Ny+j] = minmod3(s*(GH(hh,ip1,j)-GH(hh,i,j)), 0.5*(GH(hh,ip1,j)-GH(hh,im1,j)),
                                s*(GH(hh,i,j)-GH(hh,im1,j)));
          d2y[i*Ny+j] = minmod3(s*(GH(hh,i,jp1)-GH(hh,i,j)), 0.5*(GH(hh,i,jp1)-GH(hh,i,jm1)),
                                s*(GH(hh,i,j)-GH(hh,i,jm1)));
        }
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
        {
          int im1 = (i+Nx-1) % Nx, jm1 = (j+Ny-1) % Ny;
          double xm = GH(hh,im1,j) + 0.5*d2x[im1*Ny+j];
          double xp = GH(hh,i,j) - 0.5*d2x[i*Ny+j];
          double ym = GH(hh,i,jm1) + 0.5*d2y[i*Ny+jm1];
          double yp = GH(hh,i,j) + 0.5*d2y[i*Ny+j];
          A(hw_,G+i,G+j) = (GH(uu,i,j) > 0) ? xm : xp;
          A(hs_,G+i,G+j) = (GH(vv,i,j) > 0) ? ym : yp;
        }
      free(d2x); free(d2y);
    }
    xch(m,hw_,K_SCALAR);
    xch(m,hs_,K_SCALAR);
  }
#undef GH
}

/* pressure.c:570-606 */
static void build_rhs (orc_model * m)
{
  int i,j,k;
  f2_zero(&m->rhs);
  load_state(m);
  face_thickness_global(m);
  for (k = 0; k < m->L; k ++)
    for (i = G; i < G+m->Nx; i ++)
      for (j = G; j < G+m->Ny; j ++)
      {
        double hw0 = A(&m->u[k],i,j) * A(&m->hwest[k],i,j);
        double hw1 = A(&m->u[k],i+1,j) * A(&m->hwest[k],i+1,j);
        double hs0 = A(&m->v[k],i,j) * A(&m->hsouth[k],i,j);
        double hs1 = A(&m->v[k],i,j+1) * A(&m->hsouth[k],i,j+1);
        A(&m->rhs,i,j) += (hw1 - hw0) / (m->dx * m->c.dt) + (hs1 - hs0) / (m->dy * m->c.dt);
      }
  xch(m,&m->rhs,K_SCALAR);
  subtract_mean(m,&m->rhs);
  xch(m,&m->rhs,K_SCALAR);
}

/* pressure.c:609-637 */
static double op_w (orc_model * m, int i, int j)
{
  int gi = i - G;
  if (m->c.wall_ew && ((gi == 0) || (gi == m->Nx))) return 0;
  return A(&m->Hw,i,j) / SQ(m->dx);
}

static double op_s (orc_model * m, int i, int j)
{
  int gj = j - G;
  if (m->c.wall_ns && ((gj == 0) || (gj == m->Ny))) return 0;
  return A(&m->Hs,i,j) / SQ(m->dy);
}

/* pressure.c:743-814 */
static int solve_sor (orc_model * m)
{
  int iters = 0, i, j, color;
  double gmax = m->c.pi_tol + 1;
  F2 * pi = &m->pi;
  while ((gmax > m->c.pi_tol) && (iters < m->c.maxiters))
  {
    double itmax = 0;
    for (color = 0; color < 2; color ++)
    {
      double cmax = 0;
      xch(m,pi,K_SCALAR);
      for (i = G; i < G+m->Nx; i ++)
        for (j = G; j < G+m->Ny; j ++)
        {
          double Ow, Oe, Os, On, Osum, prev, nw;
          if ((((i-G)+(j-G)) & 1) != color) continue;
          Ow = op_w(m,i,j); Oe = op_w(m,i+1,j); Os = op_s(m,i,j); On = op_s(m,i,j+1);
          Osum = Ow + Oe + Os + On;
          if (Osum == 0) continue;
          prev = A(pi,i,j);
          nw = (1-m->c.sor_rp)*prev
             + m->c.sor_rp / Osum
             * (On*A(pi,i,j+1) + Os*A(pi,i,j-1) + Oe*A(pi,i+1,j) + Ow*A(pi,i-1,j)
              - A(&m->rhs,i,j));
          A(pi,i,j) = nw;
          cmax = fmax(cmax,fabs(nw-prev));
        }
      itmax = fmax(itmax,cmax);
    }
    gmax = itmax;
    iters ++;
  }
  subtract_mean(m,pi);
  xch(m,pi,K_SCALAR);
  return iters;
}

/* ------------------------------------------------- serial multigrid (MG) */

#define MGI(l,a,i,j) ((l)->a[(size_t) (i)*(l)->Ny + (j)])

static int coarsen (int n) { return (n > 1) ? (n+1)/2 : 1; }

/* multigrid.c:651-668 and 681-740 */
static void mg_restrict (const mg_level * f, const double * pf, const mg_level * c, double * pc)
{
  int ic,jc;
  if (f->power2)
  {
    for (ic = 0; ic < f->Nx/2; ic ++)
      for (jc = 0; jc < f->Ny/2; jc ++)
        pc[(size_t) ic*c->Ny+jc] = 0.25 * (pf[(size_t) (2*ic)*f->Ny+2*jc] + pf[(size_t) (2*ic+1)*f->Ny+2*jc]
                                         + pf[(size_t) (2*ic)*f->Ny+2*jc+1] + pf[(size_t) (2*ic+1)*f->Ny+2*jc+1]);
    return;
  }
  memset(pc,0,(size_t) c->Nx*c->Ny*sizeof(double));
  for (ic = 0; ic < c->Nx; ic ++)
  {
    double x0 = ((double) ic) * f->Nx / c->Nx, x1 = ((double) (ic+1)) * f->Nx / c->Nx;
    for (jc = 0; jc < c->Ny; jc ++)
    {
      double y0 = ((double) jc) * f->Ny / c->Ny, y1 = ((double) (jc+1)) * f->Ny / c->Ny;
      double wsum = 0;
      unsigned fi,fj;
      for (fi = (unsigned) floor(x0); fi < (unsigned) ceil(x1); fi ++)
      {
        double wx = fmin(x1,(double) (fi+1)) - fmax(x0,(double) fi);
        if (wx <= 0) continue;
        for (fj = (unsigned) floor(y0); fj < (unsigned) ceil(y1); fj ++)
        {
          double wy = fmin(y1,(double) (fj+1)) - fmax(y0,(double) fj), w;
          if (wy <= 0) continue;
          w = wx * wy;
          pc[(size_t) ic*c->Ny+jc] += w * pf[(size_t) fi*f->Ny+fj];
          wsum += w;
        }
      }
      if (wsum > 0) pc[(size_t) ic*c->Ny+jc] /= wsum;
    }
  }
}

static int interp_index (int idx, int N, int wall)
{
  if (N <= 1) return 0;
  if (wall)
  {
    if (idx < 0) return 0;
    if (idx >= N) return N-1;
    return idx;
  }
  return (idx + N) % N;
}

/* multigrid.c:827-932 */
static void mg_interpolate (orc_model * m, const mg_level * f, double * pf, const mg_level * c, const double * pc)
{
  int i,j;
  if (f->power2)
  {
    int hx = f->Nx/2, hy = f->Ny/2;
    for (i = 0; i < f->Nx; i ++)
    {
      int ip = (((i+1)-(i+1)%2)/2 + hx) % hx;
      int im = (ip-1 + hx) % hx;
      for (j = 0; j < f->Ny; j ++)
      {
        int jp = (((j+1)-(j+1)%2)/2 + hy) % hy;
        int jm = (jp-1 + hy) % hy;
        pf[(size_t) i*f->Ny+j] = MGI(f,wmm,i,j)*pc[(size_t) im*c->Ny+jm] + MGI(f,wpm,i,j)*pc[(size_t) ip*c->Ny+jm]
                               + MGI(f,wmp,i,j)*pc[(size_t) im*c->Ny+jp] + MGI(f,wpp,i,j)*pc[(size_t) ip*c->Ny+jp];
      }
    }
    return;
  }
  for (i = 0; i < f->Nx; i ++)
  {
    double x = (((double) i) + 0.5) * c->Nx / f->Nx - 0.5, tx;
    int imr, im, ip;
    if (m->c.wall_ew && (x <= 0)) { imr = 0; tx = 0; }
    else if (m->c.wall_ew && (x >= c->Nx-1)) { imr = c->Nx-1; tx = 0; }
    else { imr = (int) floor(x); tx = x - imr; }
    im = interp_index(imr,c->Nx,m->c.wall_ew);
    ip = interp_index(imr+1,c->Nx,m->c.wall_ew);
    for (j = 0; j < f->Ny; j ++)
    {
      double y = (((double) j) + 0.5) * c->Ny / f->Ny - 0.5, ty;
      int jmr, jm, jp;
      if (m->c.wall_ns && (y <= 0)) { jmr = 0; ty = 0; }
      else if (m->c.wall_ns && (y >= c->Ny-1)) { jmr = c->Ny-1; ty = 0; }
      else { jmr = (int) floor(y); ty = y - jmr; }
      jm = interp_index(jmr,c->Ny,m->c.wall_ns);
      jp = interp_index(jmr+1,c->Ny,m->c.wall_ns);
      pf[(size_t) i*f->Ny+j] = (1-tx)*(1-ty)*pc[(size_t) im*c->Ny+jm]
                             + tx*(1-ty)*pc[(size_t) ip*c->Ny+jm]
                             + (1-tx)*ty*pc[(size_t) im*c->Ny+jp]
                             + tx*ty*pc[(size_t) ip*c->Ny+jp];
    }
  }
}

/* multigrid.c:196-446 */
static int mg_init (orc_model * m)
{
  int Nx = m->Nx, Ny = m->Ny, nx, ny, lv, i, j;
  int wew = m->c.wall_ew, wns = m->c.wall_ns;
  m->Ngrids = 1;
  nx = Nx; ny = Ny;
  while ((nx > 1) || (ny > 1)) { nx = coarsen(nx); ny = coarsen(ny); m->Ngrids ++; }
  m->Fmg = (double *) calloc((size_t) ((Nx > Ny) ? Nx : Ny) + 1,sizeof(double));
  m->mg = (mg_level *) calloc((size_t) m->Ngrids,sizeof(mg_level));
  nx = Nx; ny = Ny;
  for (lv = m->Ngrids-1; lv >= 0; lv --)
  {
    m->mg[lv].Nx = nx; m->mg[lv].Ny = ny;
    m->mg[lv].dx = m->c.Lx/nx; m->mg[lv].dy = m->c.Ly/ny;
    nx = coarsen(nx); ny = coarsen(ny);
  }
  for (lv = m->Ngrids-1; lv > 0; lv --)
    m->mg[lv].power2 = (m->mg[lv].Nx == 2*m->mg[lv-1].Nx) && (m->mg[lv].Ny == 2*m->mg[lv-1].Ny);
  for (lv = m->Ngrids-1; lv >= 0; lv --)
  {
    mg_level * l = &m->mg[lv];
    size_t n = (size_t) l->Nx*l->Ny;
    int lx = l->Nx, ly = l->Ny;
    l->pi_temp = calloc(n,sizeof(double)); l->Hc = calloc(n,sizeof(double));
    l->Hw = calloc(n,sizeof(double)); l->Hs = calloc(n,sizeof(double));
    l->Ow = calloc(n,sizeof(double)); l->Os = calloc(n,sizeof(double));
    l->Osum = calloc(n,sizeof(double)); l->rOsum = calloc(n,sizeof(double));
    l->wmm = calloc(n,sizeof(double)); l->wmp = calloc(n,sizeof(double));
    l->wpm = calloc(n,sizeof(double)); l->wpp = calloc(n,sizeof(double));
    if (lv < m->Ngrids-1)
    {
      l->pi = calloc(n,sizeof(double)); l->rhs = calloc(n,sizeof(double)); l->own_pi = 1;
    }
    else
    {
      l->pi = calloc(n,sizeof(double)); l->rhs = calloc(n,sizeof(double)); l->own_pi = 1;
    }
    if (lv == m->Ngrids-1)
    {
      for (i = 0; i < Nx; i ++)
        for (j = 0; j < Ny; j ++)
          MGI(l,Hc,i,j) = A(&m->Hc,G+i,G+j);
    }
    else
    {
      mg_restrict(&m->mg[lv+1],m->mg[lv+1].Hc,l,l->Hc);
    }
    for (i = 0; i < lx; i ++)
    {
      int im1 = (i+lx-1) % lx;
      for (j = 0; j < ly; j ++)
      {
        int jm1 = (j+ly-1) % ly;
        MGI(l,Hw,i,j) = 0.5 * (MGI(l,Hc,i,j)+MGI(l,Hc,im1,j));
        MGI(l,Hs,i,j) = 0.5 * (MGI(l,Hc,i,j)+MGI(l,Hc,i,jm1));
      }
    }
    for (i = 0; i < lx; i ++)
    {
      for (j = 0; j < ly; j ++) MGI(l,Os,i,j) = MGI(l,Hs,i,j) / SQ(l->dy);
      if (wns) MGI(l,Os,i,0) = 0;
    }
    for (j = 0; j < ly; j ++)
    {
      for (i = 0; i < lx; i ++) MGI(l,Ow,i,j) = MGI(l,Hw,i,j) / SQ(l->dx);
      if (wew) MGI(l,Ow,0,j) = 0;
    }
    for (i = 0; i < lx; i ++)
    {
      int ip1 = (i + lx + 1) % lx;
      for (j = 0; j < ly; j ++)
      {
        int jp1 = (j + ly + 1) % ly;
        MGI(l,Osum,i,j) = MGI(l,Ow,i,j) + MGI(l,Ow,ip1,j) + MGI(l,Os,i,j) + MGI(l,Os,i,jp1);
        MGI(l,rOsum,i,j) = 1 / MGI(l,Osum,i,j);
      }
    }
    for (i = 0; i < lx; i ++)
      for (j = 0; j < ly; j ++)
      {
        double ai = (i%2==1) ? 0.75 : 0.25, bi = (i%2==1) ? 0.25 : 0.75;
        double aj = (j%2==1) ? 0.75 : 0.25, bj = (j%2==1) ? 0.25 : 0.75;
        MGI(l,wmm,i,j) = ai * aj;
        MGI(l,wmp,i,j) = ai * bj;
        MGI(l,wpm,i,j) = bi * aj;
        MGI(l,wpp,i,j) = bi * bj;
      }
    if (wns)
    {
      for (i = 0; i < lx; i ++)
      {
        MGI(l,wmm,i,0) = 0; MGI(l,wpm,i,0) = 0;
        MGI(l,wmp,i,0) = (i%2==1) ? 0.75 : 0.25; MGI(l,wpp,i,0) = (i%2==1) ? 0.25 : 0.75;
        MGI(l,wmp,i,ly-1) = 0; MGI(l,wpp,i,ly-1) = 0;
        MGI(l,wmm,i,ly-1) = (i%2==1) ? 0.75 : 0.25; MGI(l,wpm,i,ly-1) = (i%2==1) ? 0.25 : 0.75;
      }
    }
    if (wew)
    {
      for (j = 0; j < ly; j ++)
      {
        MGI(l,wmm,0,j) = 0; MGI(l,wmp,0,j) = 0;
        MGI(l,wpm,0,j) = (j%2==1) ? 0.75 : 0.25; MGI(l,wpp,0,j) = (j%2==1) ? 0.25 : 0.75;
        MGI(l,wpm,lx-1,j) = 0; MGI(l,wpp,lx-1,j) = 0;
        MGI(l,wmm,lx-1,j) = (j%2==1) ? 0.75 : 0.25; MGI(l,wmp,lx-1,j) = (j%2==1) ? 0.25 : 0.75;
      }
    }
    if (wns && wew)
    {
      MGI(l,wmm,0,0) = 0; MGI(l,wmp,0,0) = 0; MGI(l,wpm,0,0) = 0; MGI(l,wpp,0,0) = 1;
      MGI(l,wmm,0,ly-1) = 0; MGI(l,wmp,0,ly-1) = 0; MGI(l,wpm,0,ly-1) = 1; MGI(l,wpp,0,ly-1) = 0;
      MGI(l,wmm,lx-1,0) = 0; MGI(l,wmp,lx-1,0) = 1; MGI(l,wpm,lx-1,0) = 0; MGI(l,wpp,lx-1,0) = 0;
      MGI(l,wmm,lx-1,ly-1) = 1; MGI(l,wmp,lx-1,ly-1) = 0; MGI(l,wpm,lx-1,ly-1) = 0; MGI(l,wpp,lx-1,ly-1) = 0;
    }
  }
  m->mg_ready = 1;
  return 0;
}

/* multigrid.c:461-511 */
static void mg_exact (orc_model * m, mg_level * l)
{
  int i,j;
  if ((l->Nx == 1) && (l->Ny == 1)) { l->pi[0] = 0; return; }
  if (l->Nx == 1)
  {
    m->Fmg[0] = 0;
    for (j = 1; j <= l->Ny; j ++) m->Fmg[j] = m->Fmg[j-1] + l->rhs[j-1];
    l->pi[0] = 0;
    for (j = 1; j < l->Ny; j ++) l->pi[j] = l->pi[j-1] + m->Fmg[j]/l->Os[j];
  }
  else
  {
    m->Fmg[0] = 0;
    for (i = 1; i <= l->Nx; i ++) m->Fmg[i] = m->Fmg[i-1] + l->rhs[(size_t) (i-1)*l->Ny];
    l->pi[0] = 0;
    for (i = 1; i < l->Nx; i ++) l->pi[(size_t) i*l->Ny] = l->pi[(size_t) (i-1)*l->Ny] + m->Fmg[i]/l->Ow[(size_t) i*l->Ny];
  }
}

/* multigrid.c:536-568: damped sweep, updated in place in lexicographic order */
static void mg_relax (orc_model * m, mg_level * l)
{
  int i,j,Nx = l->Nx,Ny = l->Ny;
  double w = m->c.omega_mg;
  for (i = 0; i < Nx; i ++)
  {
    int im1 = (i+Nx-1) % Nx, ip1 = (i+Nx+1) % Nx;
    for (j = 0; j < Ny; j ++)
    {
      int jm1 = (j+Ny-1) % Ny, jp1 = (j+Ny+1) % Ny;
      MGI(l,pi,i,j) = w * MGI(l,rOsum,i,j) * ( MGI(l,Os,i,jp1)*MGI(l,pi,i,jp1) + MGI(l,Os,i,j)*MGI(l,pi,i,jm1)
                    + MGI(l,Ow,ip1,j)*MGI(l,pi,ip1,j) + MGI(l,Ow,i,j)*MGI(l,pi,im1,j) - MGI(l,rhs,i,j) )
                    + (1-w) * MGI(l,pi,i,j);
    }
  }
}

/* multigrid.c:599-627 */
static void mg_residual (mg_level * l, double * res)
{
  int i,j,Nx = l->Nx,Ny = l->Ny;
  for (i = 0; i < Nx; i ++)
  {
    int im1 = (i+Nx-1) % Nx, ip1 = (i+Nx+1) % Nx;
    for (j = 0; j < Ny; j ++)
    {
      int jm1 = (j+Ny-1) % Ny, jp1 = (j+Ny+1) % Ny;
      res[(size_t) i*Ny+j] = MGI(l,Os,i,jp1)*MGI(l,pi,i,jp1) + MGI(l,Os,i,j)*MGI(l,pi,i,jm1)
                           + MGI(l,Ow,ip1,j)*MGI(l,pi,ip1,j) + MGI(l,Ow,i,j)*MGI(l,pi,im1,j)
                           - MGI(l,Osum,i,j)*MGI(l,pi,i,j) - MGI(l,rhs,i,j);
    }
  }
}

/* multigrid.c:1123-1156 */
static double mg_max_residual (mg_level * l)
{
  int i,j,Nx = l->Nx,Ny = l->Ny;
  double mx = 0;
  for (i = 0; i < Nx; i ++)
  {
    int im1 = (i+Nx-1) % Nx, ip1 = (i+Nx+1) % Nx;
    for (j = 0; j < Ny; j ++)
    {
      int jm1 = (j+Ny-1) % Ny, jp1 = (j+Ny+1) % Ny;
      double r = MGI(l,pi,i,j) - MGI(l,rOsum,i,j) * ( MGI(l,Os,i,jp1)*MGI(l,pi,i,jp1) + MGI(l,Os,i,j)*MGI(l,pi,i,jm1)
               + MGI(l,Ow,ip1,j)*MGI(l,pi,ip1,j) + MGI(l,Ow,i,j)*MGI(l,pi,im1,j) - MGI(l,rhs,i,j) );
      mx = fmax(mx,fabs(r));
    }
  }
  return mx;
}

/* multigrid.c:1023-1096 */
static void mg_vcycle (orc_model * m, int n)
{
  mg_level * l = &m->mg[n];
  size_t i, nn = (size_t) l->Nx*l->Ny;
  if (n == 0) { mg_exact(m,l); return; }
  mg_relax(m,l);
  mg_residual(l,l->pi_temp);
  mg_restrict(l,l->pi_temp,&m->mg[n-1],m->mg[n-1].rhs);
  memset(m->mg[n-1].pi,0,(size_t) m->mg[n-1].Nx*m->mg[n-1].Ny*sizeof(double));
  mg_vcycle(m,n-1);
  mg_interpolate(m,l,l->pi_temp,&m->mg[n-1],m->mg[n-1].pi);
  for (i = 0; i < nn; i ++) l->pi[i] -= l->pi_temp[i];
  mg_relax(m,l);
}

/* multigrid.c:1172-1213 */
static int mg_iterate (orc_model * m, int n)
{
  int iters = 0;
  double mx = m->c.pi_tol + 1;
  while ((mx > m->c.pi_tol) && (iters < m->c.maxiters))
  {
    mg_vcycle(m,n);
    mx = mg_max_residual(&m->mg[n]);
    iters ++;
  }
  return iters;
}

/* pressure.c:820-914 + multigrid.c:1236-1343; the mean of pi is not removed */
static int solve_mg (orc_model * m)
{
  int i,j,iters,n;
  mg_level * f;
  if (!m->mg_ready) mg_init(m);
  f = &m->mg[m->Ngrids-1];
  for (i = 0; i < m->Nx; i ++)
    for (j = 0; j < m->Ny; j ++)
    {
      MGI(f,pi,i,j) = A(&m->pi,G+i,G+j);
      MGI(f,rhs,i,j) = A(&m->rhs,G+i,G+j);
    }
  if (m->c.use_full_mg)
  {
    for (n = m->Ngrids-1; n > 0; n --) mg_restrict(&m->mg[n],m->mg[n].rhs,&m->mg[n-1],m->mg[n-1].rhs);
    mg_vcycle(m,0);
    iters = 0;
    for (n = 1; n < m->Ngrids; n ++)
    {
      mg_interpolate(m,&m->mg[n],m->mg[n].pi,&m->mg[n-1],m->mg[n-1].pi);
      iters = mg_iterate(m,n);
    }
  }
  else
  {
    iters = mg_iterate(m,m->Ngrids-1);
  }
  for (i = 0; i < m->Nx; i ++)
    for (j = 0; j < m->Ny; j ++)
      A(&m->pi,G+i,G+j) = MGI(f,pi,i,j);
  xch(m,&m->pi,K_SCALAR);
  return iters;
}

/* pressure.c:652-690 */
static void residual_norms (orc_model * m)
{
  int i,j;
  double mx = 0, ss = 0;
  xch(m,&m->pi,K_SCALAR);
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
    {
      double Ow = op_w(m,i,j), Oe = op_w(m,i+1,j), Os = op_s(m,i,j), On = op_s(m,i,j+1);
      double pc = A(&m->pi,i,j);
      double Lp = Oe*(A(&m->pi,i+1,j)-pc) + Ow*(A(&m->pi,i-1,j)-pc)
                + On*(A(&m->pi,i,j+1)-pc) + Os*(A(&m->pi,i,j-1)-pc);
      double r = A(&m->rhs,i,j) - Lp;
      mx = fmax(mx,fabs(r));
      ss += r*r;
    }
  m->last.residual_max = mx;
  m->last.residual_rms = sqrt(ss / ((double) m->Nx * (double) m->Ny));
}

/* pressure.c:693-737 */
static void divergence_norms (orc_model * m)
{
  int i,j,k;
  double mx = 0, ss = 0;
  load_state(m);
  face_thickness_global(m);
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
    {
      double dv = 0;
      for (k = 0; k < m->L; k ++)
      {
        double hw0 = A(&m->u[k],i,j) * A(&m->hwest[k],i,j);
        double hw1 = A(&m->u[k],i+1,j) * A(&m->hwest[k],i+1,j);
        double hs0 = A(&m->v[k],i,j) * A(&m->hsouth[k],i,j);
        double hs1 = A(&m->v[k],i,j+1) * A(&m->hsouth[k],i,j+1);
        dv += (hw1 - hw0) / m->dx + (hs1 - hs0) / m->dy;
      }
      mx = fmax(mx,fabs(dv));
      ss += dv*dv;
    }
  m->last.div_max = mx;
  m->last.div_rms = sqrt(ss / ((double) m->Nx * (double) m->Ny));
}

/* pressure.c:2182-2248 (budget diagnostics omitted) */
static void apply_correction (orc_model * m)
{
  int i,j,k;
  double dt = m->c.dt;
  for (k = 0; k < m->L; k ++)
  {
    for (i = G; i < G+m->Nx; i ++)
    {
      if (m->c.wall_ew && (i == G)) continue;
      for (j = G; j < G+m->Ny; j ++)
        A(&m->u[k],i,j) += -dt * (A(&m->pi,i,j) - A(&m->pi,i-1,j)) / m->dx;
    }
    for (j = G; j < G+m->Ny; j ++)
    {
      if (m->c.wall_ns && (j == G)) continue;
      for (i = G; i < G+m->Nx; i ++)
        A(&m->v[k],i,j) += -dt * (A(&m->pi,i,j) - A(&m->pi,i,j-1)) / m->dy;
    }
  }
  state_halos(m,m->u,m->v,m->h);
}

/* ------------------------------------- distributed multigrid, serial build (DMG) */

/* pressure.c:916-2176 with one rank: every level is one tile, transfers are the local
 * 2:1 ones, and the last level (a side <= 8 or odd) is solved by the serial red-black SOR
 * of the gathered tail. */
#define DMG_PRE 3
#define DMG_POST 3
#define DMG_MIN 8
#define DMG_MAXL 32

typedef struct
{
  int Nx, Ny;
  double dx, dy;
  F2 x, rhs, res, Hc, Hw, Hs;
} dmg_level;

static double dmg_ow (orc_model * m, const dmg_level * l, int i, int j)
{
  int gi = i - G;
  if (m->c.wall_ew && ((gi == 0) || (gi == l->Nx))) return 0;
  return A(&l->Hw,i,j) / SQ(l->dx);
}

static double dmg_os (orc_model * m, const dmg_level * l, int i, int j)
{
  int gj = j - G;
  if (m->c.wall_ns && ((gj == 0) || (gj == l->Ny))) return 0;
  return A(&l->Hs,i,j) / SQ(l->dy);
}

/* pressure.c:1387-1438: in-place weighted sweeps (x outer, y inner) whose halo comes from
 * the previous sweep; returns the largest update of the last sweep */
static double dmg_smooth (orc_model * m, dmg_level * l, int nsweeps)
{
  int sweep,i,j;
  double gmax = 0;
  for (sweep = 0; sweep < nsweeps; sweep ++)
  {
    double lmax = 0;
    xch(m,&l->x,K_SCALAR);
    for (i = G; i < G+l->Nx; i ++)
      for (j = G; j < G+l->Ny; j ++)
      {
        double Ow = dmg_ow(m,l,i,j), Oe = dmg_ow(m,l,i+1,j), Os = dmg_os(m,l,i,j), On = dmg_os(m,l,i,j+1);
        double Osum = Ow + Oe + Os + On, xo, xj, xn;
        if (Osum == 0) continue;
        xo = A(&l->x,i,j);
        xj = (Oe*A(&l->x,i+1,j) + Ow*A(&l->x,i-1,j) + On*A(&l->x,i,j+1) + Os*A(&l->x,i,j-1)
            - A(&l->rhs,i,j)) / Osum;
        xn = xo + m->c.omega_mg*(xj-xo);
        A(&l->x,i,j) = xn;
        lmax = fmax(lmax,fabs(xn-xo));
      }
    gmax = lmax;
  }
  xch(m,&l->x,K_SCALAR);
  return gmax;
}

/* pressure.c:1441-1466: res = rhs - L(x) */
static void dmg_residual (orc_model * m, dmg_level * l)
{
  int i,j;
  xch(m,&l->x,K_SCALAR);
  for (i = G; i < G+l->Nx; i ++)
    for (j = G; j < G+l->Ny; j ++)
    {
      double Ow = dmg_ow(m,l,i,j), Oe = dmg_ow(m,l,i+1,j), Os = dmg_os(m,l,i,j), On = dmg_os(m,l,i,j+1);
      double xc = A(&l->x,i,j);
      A(&l->res,i,j) = A(&l->rhs,i,j)
                     - (Oe*(A(&l->x,i+1,j)-xc) + Ow*(A(&l->x,i-1,j)-xc)
                      + On*(A(&l->x,i,j+1)-xc) + Os*(A(&l->x,i,j-1)-xc));
    }
  xch(m,&l->res,K_SCALAR);
}

/* pressure.c:1469-1544: kind 0 = 2x2 mean, 1 = west faces (y pair), 2 = south faces (x pair) */
static void dmg_restrict (orc_model * m, F2 * c, const F2 * f, int cNx, int cNy, int kind)
{
  int i,j;
  f2_zero(c);
  for (i = 0; i < cNx; i ++)
    for (j = 0; j < cNy; j ++)
    {
      int a = 2*i + G, b = 2*j + G;
      if (kind == 0)
        A(c,i+G,j+G) = 0.25*(A(f,a,b) + A(f,a+1,b) + A(f,a,b+1) + A(f,a+1,b+1));
      else if (kind == 1)
        A(c,i+G,j+G) = 0.5*(A(f,a,b) + A(f,a,b+1));
      else
        A(c,i+G,j+G) = 0.5*(A(f,a,b) + A(f,a+1,b));
    }
  xch(m,c,K_SCALAR);
}

/* pressure.c:1547-1600: fine x += bilinear(coarse x); returns max |correction| */
static double dmg_prolong (orc_model * m, dmg_level * f, dmg_level * c)
{
  int i,j;
  double mx = 0;
  xch(m,&c->x,K_SCALAR);
  for (i = 0; i < c->Nx; i ++)
    for (j = 0; j < c->Ny; j ++)
    {
      int ic = i+G, jc = j+G, a = 2*i+G, b = 2*j+G;
      F2 * X = &c->x;
      double e_sw = 0.5625*A(X,ic,jc) + 0.1875*A(X,ic-1,jc) + 0.1875*A(X,ic,jc-1) + 0.0625*A(X,ic-1,jc-1);
      double e_se = 0.5625*A(X,ic,jc) + 0.1875*A(X,ic+1,jc) + 0.1875*A(X,ic,jc-1) + 0.0625*A(X,ic+1,jc-1);
      double e_nw = 0.5625*A(X,ic,jc) + 0.1875*A(X,ic-1,jc) + 0.1875*A(X,ic,jc+1) + 0.0625*A(X,ic-1,jc+1);
      double e_ne = 0.5625*A(X,ic,jc) + 0.1875*A(X,ic+1,jc) + 0.1875*A(X,ic,jc+1) + 0.0625*A(X,ic+1,jc+1);
      A(&f->x,a,b) += e_sw;
      A(&f->x,a+1,b) += e_se;
      A(&f->x,a,b+1) += e_nw;
      A(&f->x,a+1,b+1) += e_ne;
      mx = fmax(mx,fabs(e_sw));
      mx = fmax(mx,fabs(e_se));
      mx = fmax(mx,fabs(e_nw));
      mx = fmax(mx,fabs(e_ne));
    }
  xch(m,&f->x,K_SCALAR);
  return mx;
}

/* pressure.c:360-437 and 1713-1780: serial red-black SOR of the last level from its Hc
 * (faces averaged with modular indices, wall faces zeroed); the mean is removed at the
 * end. Its own updates do not enter the V-cycle's measure. */
static void dmg_tail (orc_model * m, dmg_level * l)
{
  int Nx = l->Nx, Ny = l->Ny, i, j, color, iters = 0;
  double * Hw = (double *) calloc((size_t) Nx*Ny,sizeof(double));
  double * Hs = (double *) calloc((size_t) Nx*Ny,sizeof(double));
  double mu = m->c.pi_tol + 1, mean = 0, om = m->c.sor_rp;
#define HC(a,b) A(&l->Hc,G+(a),G+(b))
#define PX(a,b) A(&l->x,G+(a),G+(b))
  for (i = 0; i < Nx; i ++)
    for (j = 0; j < Ny; j ++)
    {
      int im1 = (i+Nx-1) % Nx, jm1 = (j+Ny-1) % Ny;
      Hw[(size_t) i*Ny+j] = 0.5*(HC(i,j) + HC(im1,j));
      Hs[(size_t) i*Ny+j] = 0.5*(HC(i,j) + HC(i,jm1));
    }
  if (m->c.wall_ew) for (j = 0; j < Ny; j ++) Hw[j] = 0;
  if (m->c.wall_ns) for (i = 0; i < Nx; i ++) Hs[(size_t) i*Ny] = 0;
  while ((mu > m->c.pi_tol) && (iters < m->c.maxiters))
  {
    mu = 0;
    for (color = 0; color < 2; color ++)
      for (i = 0; i < Nx; i ++)
      {
        int im1 = (i+Nx-1) % Nx, ip1 = (i+1) % Nx;
        for (j = 0; j < Ny; j ++)
        {
          int jm1 = (j+Ny-1) % Ny, jp1 = (j+1) % Ny;
          double Ow = (m->c.wall_ew && i == 0) ? 0 : Hw[(size_t) i*Ny+j] / SQ(l->dx);
          double Oe = (m->c.wall_ew && i+1 == Nx) ? 0 : Hw[(size_t) ((i+1) % Nx)*Ny+j] / SQ(l->dx);
          double Os = (m->c.wall_ns && j == 0) ? 0 : Hs[(size_t) i*Ny+j] / SQ(l->dy);
          double On = (m->c.wall_ns && j+1 == Ny) ? 0 : Hs[(size_t) i*Ny+(j+1) % Ny] / SQ(l->dy);
          double Osum = Ow + Oe + Os + On, old, nv;
          if (((i+j) & 1) != color) continue;
          if (Osum == 0) continue;
          old = PX(i,j);
          nv = (1-om)*old + om*(Oe*PX(ip1,j) + Ow*PX(im1,j) + On*PX(i,jp1) + Os*PX(i,jm1) - A(&l->rhs,G+i,G+j)) / Osum;
          PX(i,j) = nv;
          mu = fmax(mu,fabs(nv-old));
        }
      }
    iters ++;
  }
  for (i = 0; i < Nx; i ++)
    for (j = 0; j < Ny; j ++) mean += PX(i,j);
  mean /= ((double) Nx * (double) Ny);
  for (i = 0; i < Nx; i ++)
    for (j = 0; j < Ny; j ++) PX(i,j) -= mean;
#undef HC
#undef PX
  free(Hw);
  free(Hs);
  xch(m,&l->x,K_SCALAR);
}

/* pressure.c:2063-2123 */
static double dmg_vcycle (orc_model * m, dmg_level * lv, int n, int l)
{
  double mu;
  dmg_level * c;
  if (l == n-1)
  {
    dmg_tail(m,&lv[l]);
    return 0;
  }
  c = &lv[l+1];
  mu = dmg_smooth(m,&lv[l],DMG_PRE);
  dmg_residual(m,&lv[l]);
  dmg_restrict(m,&c->rhs,&lv[l].res,c->Nx,c->Ny,0);
  dmg_restrict(m,&c->Hc,&lv[l].Hc,c->Nx,c->Ny,0);
  dmg_restrict(m,&c->Hw,&lv[l].Hw,c->Nx,c->Ny,1);
  dmg_restrict(m,&c->Hs,&lv[l].Hs,c->Nx,c->Ny,2);
  f2_zero(&c->x);
  mu = fmax(mu,dmg_vcycle(m,lv,n,l+1));
  mu = fmax(mu,dmg_prolong(m,&lv[l],c));
  mu = fmax(mu,dmg_smooth(m,&lv[l],DMG_POST));
  return mu;
}

/* pressure.c:2126-2176; grids that cannot start with a clean 2:1 coarsening fall back to
 * the gathered multigrid, as the reference does */
static int solve_dmg (orc_model * m)
{
  dmg_level lv[DMG_MAXL];
  int n = 0, Nx = m->Nx, Ny = m->Ny, cycles = 0, l, i, j;
  double mu = m->c.pi_tol + 1;
  if ((Nx <= DMG_MIN) || (Ny <= DMG_MIN) || (Nx % 2) || (Ny % 2)) return solve_mg(m);
  while (n < DMG_MAXL)
  {
    dmg_level * L = &lv[n];
    L->Nx = Nx; L->Ny = Ny;
    L->dx = m->c.Lx / Nx; L->dy = m->c.Ly / Ny;
    if (!f2_alloc(&L->x,Nx,Ny) || !f2_alloc(&L->rhs,Nx,Ny) || !f2_alloc(&L->res,Nx,Ny)
     || !f2_alloc(&L->Hc,Nx,Ny) || !f2_alloc(&L->Hw,Nx,Ny) || !f2_alloc(&L->Hs,Nx,Ny))
      return -1;
    n ++;
    if ((Nx <= DMG_MIN) || (Ny <= DMG_MIN) || (Nx % 2) || (Ny % 2)) break;
    Nx = (Nx+1)/2;
    Ny = (Ny+1)/2;
  }
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++)
    {
      A(&lv[0].x,i,j) = A(&m->pi,i,j);
      A(&lv[0].rhs,i,j) = A(&m->rhs,i,j);
      A(&lv[0].Hc,i,j) = A(&m->Hc,i,j);
      A(&lv[0].Hw,i,j) = A(&m->Hw,i,j);
      A(&lv[0].Hs,i,j) = A(&m->Hs,i,j);
    }
  xch(m,&lv[0].x,K_SCALAR);
  xch(m,&lv[0].rhs,K_SCALAR);
  xch(m,&lv[0].Hc,K_SCALAR);
  xch(m,&lv[0].Hw,K_SCALAR);
  xch(m,&lv[0].Hs,K_SCALAR);
  while ((mu > m->c.pi_tol) && (cycles < m->c.maxiters))
  {
    mu = dmg_vcycle(m,lv,n,0);
    subtract_mean(m,&lv[0].x);
    cycles ++;
  }
  for (i = G; i < G+m->Nx; i ++)
    for (j = G; j < G+m->Ny; j ++) A(&m->pi,i,j) = A(&lv[0].x,i,j);
  for (l = 0; l < n; l ++)
  {
    free(lv[l].x.d); free(lv[l].rhs.d); free(lv[l].res.d);
    free(lv[l].Hc.d); free(lv[l].Hw.d); free(lv[l].Hs.d);
  }
  subtract_mean(m,&m->pi);
  xch(m,&m->pi,K_SCALAR);
  return cycles;
}

int orc_pressure (orc_model * m, int update_diags, orc_pstats * st)
{
  int iters;
  (void) update_diags;
  if (!m->c.use_rl) { if (st) memset(st,0,sizeof(*st)); return 0; }
  static_geometry(m);
  correct_thickness(m);
  build_rhs(m);
  if (m->c.solver == 1) iters = solve_mg(m);
  else if (m->c.solver == 2) iters = solve_dmg(m);
  else iters = solve_sor(m);
  if (m->c.pressure_timing) residual_norms(m);
  apply_correction(m);
  if (m->c.pressure_timing) divergence_norms(m);
  m->last.iters = iters;
  if (st) *st = m->last;
  return iters;
}

/* pawsim.c:266-304 */
int orc_prelim (orc_model * m, orc_pstats * st)
{
  load_state(m);
  static_geometry(m);
  forcing_update(m,m->t);
  core(m);
  if (m->c.use_rl)
  {
    int it = orc_pressure(m,0,st);
    if (it < 0) return it;
    load_state(m);
    static_geometry(m);
    forcing_update(m,m->t);
    core(m);
  }
  return 0;
}

int orc_run_steps (orc_model * m, int n0, int nsteps, orc_pstats * last)
{
  int n;
  for (n = n0; n < n0 + nsteps; n ++)
  {
    orc_integrator_step(m,n);
    if (m->c.use_rl)
    {
      int it = orc_pressure(m,1,last);
      if (it < 0) return it;
    }
  }
  return 0;
}

double orc_time (const orc_model * m)
{
  return m->t;
}

/* diagnostics.c:478-700: kinetic and potential energy of the whole domain and the potential
 * enstrophy of each layer, summed in the reference's serial order (layer, then x, then y).
 * h, u, v are the state (halos current); eta is built from the thickness last copied into
 * the work arrays, which `reload` refreshes first, as the online averages do every step. */
int orc_energy (orc_model * m, int reload, double * ke, double * pe, double * z)
{
  int i,j,k;
  const double dx = m->dx, dy = m->dy;
  double KE = 0, PE = 0;
  if (reload) load_state(m);
  calc_eta(m);
  for (k = 0; k < m->L; k ++)
  {
    const F2 * h = &m->h[k], * u = &m->u[k], * v = &m->v[k];
    double Z = 0;
    for (i = G; i < G+m->Nx; i ++)
    {
      const int gi = i - G;
      for (j = G; j < G+m->Ny; j ++)
      {
        const int gj = j - G;
        double hq, zeta, pv, ked = 0, gtot;
        if (m->c.wall_ns && gj == 0)
        {
          hq = 0.5*(A(h,i-1,j) + A(h,i,j));
          zeta = 0;
        }
        else if (m->c.wall_ew && gi == 0)
        {
          hq = 0.5*(A(h,i,j-1) + A(h,i,j));
          zeta = 0;
        }
        else
        {
          hq = 0.25*(A(h,i,j) + A(h,i-1,j-1) + A(h,i-1,j) + A(h,i,j-1));
          zeta = (A(u,i,j-1) - A(u,i,j)) / dy + (A(v,i,j) - A(v,i-1,j)) / dx;
        }
        if (hq != 0)
        {
          pv = (2*A(&m->omz,i,j) + zeta) / hq;
          Z += dx*dy * 0.5 * hq * SQ(pv);
        }
        if (m->c.thick_scheme == 1)
        {
          /* HK83 (diagnostics.c:577-642) */
          ked = 0;
          if (m->c.wall_ns && gj == 0)
            ked += (A(h,i,j)+A(h,i+1,j)) * (1.25*SQ(A(u,i+1,j)) + 0.25*SQ(A(u,i+1,j+1)))
                 + (A(h,i-1,j)+A(h,i,j)) * (1.25*SQ(A(u,i,j)) + 0.25*SQ(A(u,i,j+1)));
          else if (m->c.wall_ns && gj == m->Ny-1)
            ked += (A(h,i,j)+A(h,i+1,j)) * (1.25*SQ(A(u,i+1,j)) + 0.25*SQ(A(u,i+1,j-1)))
                 + (A(h,i-1,j)+A(h,i,j)) * (1.25*SQ(A(u,i,j)) + 0.25*SQ(A(u,i,j-1)));
          else
            ked += (A(h,i,j)+A(h,i+1,j)) * (SQ(A(u,i+1,j)) + 0.25*SQ(A(u,i+1,j+1)) + 0.25*SQ(A(u,i+1,j-1)))
                 + (A(h,i-1,j)+A(h,i,j)) * (SQ(A(u,i,j)) + 0.25*SQ(A(u,i,j+1)) + 0.25*SQ(A(u,i,j-1)));
          if (m->c.wall_ew && gi == 0)
            ked += (A(h,i,j)+A(h,i,j+1)) * (1.25*SQ(A(v,i,j+1)) + 0.25*SQ(A(v,i+1,j+1)))
                 + (A(h,i,j-1)+A(h,i,j)) * (1.25*SQ(A(v,i,j)) + 0.25*SQ(A(v,i+1,j)));
          else if (m->c.wall_ew && gi == m->Nx-1)
            ked += (A(h,i,j)+A(h,i,j+1)) * (1.25*SQ(A(v,i,j+1)) + 0.25*SQ(A(v,i-1,j+1)))
                 + (A(h,i,j-1)+A(h,i,j)) * (1.25*SQ(A(v,i,j)) + 0.25*SQ(A(v,i-1,j)));
          else
            ked += (A(h,i,j)+A(h,i,j+1)) * (SQ(A(v,i,j+1)) + 0.25*SQ(A(v,i+1,j+1)) + 0.25*SQ(A(v,i-1,j+1)))
                 + (A(h,i,j-1)+A(h,i,j)) * (SQ(A(v,i,j)) + 0.25*SQ(A(v,i+1,j)) + 0.25*SQ(A(v,i-1,j)));
          ked *= dx*dy/12.0;
        }
        else
        {
          /* AL81, UP3, KT00 (diagnostics.c:562-575) */
          ked = 0.125 * dx*dy
              * ((A(h,i,j)+A(h,i+1,j)) * SQ(A(u,i+1,j))
               + (A(h,i-1,j)+A(h,i,j)) * SQ(A(u,i,j))
               + (A(h,i,j)+A(h,i,j+1)) * SQ(A(v,i,j+1))
               + (A(h,i,j-1)+A(h,i,j)) * SQ(A(v,i,j)));
        }
        gtot = m->geff[k];
        KE += ked;
        PE += dx*dy * gtot * A(h,i,j) * (A(&m->eta[k],i,j) - 0.5*A(h,i,j));
        PE += dx*dy * gtot * (m->c.h0*m->c.h0*m->c.h0*m->c.h0) / SQ(A(h,i,j)) / 6;
      }
    }
    z[k] = Z;
  }
  *ke = KE;
  *pe = PE;
  return 0;
}

/* ------------------------------------------------------------ lifecycle */

orc_model * orc_create (const orc_cfg * cfg)
{
  orc_model * m = (orc_model *) calloc(1,sizeof(orc_model));
  int L, nx, ny, lv;
  if (m == NULL) return NULL;
  m->c = *cfg;
  L = m->L = cfg->Nlay; nx = m->Nx = cfg->Nx; ny = m->Ny = cfg->Ny;
  if ((L < 1) || (nx < 4) || (ny < 4) || (cfg->tau_nrecs < 1) || (cfg->wdia_nrecs < 1))
  {
    free(m);
    return NULL;
  }
  m->dx = cfg->Lx / nx;
  m->dy = cfg->Ly / ny;
  m->t = cfg->tmin;
  m->u = f2_alloc_n(L,nx,ny); m->v = f2_alloc_n(L,nx,ny); m->h = f2_alloc_n(L,nx,ny);
  for (lv = 0; lv < 3; lv ++)
  {
    m->tu[lv] = f2_alloc_n(L,nx,ny); m->tv[lv] = f2_alloc_n(L,nx,ny); m->th[lv] = f2_alloc_n(L,nx,ny);
  }
  f2_alloc(&m->hhs,nx,ny); f2_alloc(&m->hhb,nx,ny); f2_alloc(&m->omz,nx,ny);
  f2_alloc(&m->uLid,nx,ny); f2_alloc(&m->vLid,nx,ny); f2_alloc(&m->fbx,nx,ny);
  f2_alloc(&m->fby,nx,ny); f2_alloc(&m->hTime,nx,ny);
  m->taux = f2_alloc_n(cfg->tau_nrecs,nx,ny); m->tauy = f2_alloc_n(cfg->tau_nrecs,nx,ny);
  m->uRelax = f2_alloc_n(L,nx,ny); m->vRelax = f2_alloc_n(L,nx,ny);
  m->hRelax = f2_alloc_n(L,nx,ny); m->eRelax = f2_alloc_n(L,nx,ny);
  m->uTime = f2_alloc_n(L,nx,ny); m->vTime = f2_alloc_n(L,nx,ny); m->eTime = f2_alloc_n(L,nx,ny);
  m->wdia_ff = f2_alloc_n(cfg->wdia_nrecs*(L+1),nx,ny);
  m->nu_u = f2_alloc_n(L,nx,ny); m->nu_v = f2_alloc_n(L,nx,ny);
  m->gg = (double *) calloc((size_t) L,sizeof(double));
  m->geff = (double *) calloc((size_t) L,sizeof(double));
  m->uw = f2_alloc_n(L,nx,ny); m->vw = f2_alloc_n(L,nx,ny); m->hw = f2_alloc_n(L,nx,ny);
  m->dtu = f2_alloc_n(L,nx,ny); m->dtv = f2_alloc_n(L,nx,ny); m->dth = f2_alloc_n(L,nx,ny);
  m->hwest = f2_alloc_n(L,nx,ny); m->hsouth = f2_alloc_n(L,nx,ny);
  m->hFsw = f2_alloc_n(L,nx,ny); m->hFss = f2_alloc_n(L,nx,ny);
  m->hFbw = f2_alloc_n(L,nx,ny); m->hFbs = f2_alloc_n(L,nx,ny);
  m->hhq = f2_alloc_n(L,nx,ny); m->zeta = f2_alloc_n(L,nx,ny); m->qq = f2_alloc_n(L,nx,ny);
  m->al = f2_alloc_n(L,nx,ny); m->be = f2_alloc_n(L,nx,ny); m->ga = f2_alloc_n(L,nx,ny);
  m->de = f2_alloc_n(L,nx,ny); m->ep = f2_alloc_n(L,nx,ny); m->ph = f2_alloc_n(L,nx,ny);
  m->la = f2_alloc_n(L,nx,ny); m->mu = f2_alloc_n(L,nx,ny);
  m->pp = f2_alloc_n(L,nx,ny); m->KE = f2_alloc_n(L,nx,ny); m->MM = f2_alloc_n(L,nx,ny);
  m->eta = f2_alloc_n(L+1,nx,ny); m->wdia = f2_alloc_n(L+1,nx,ny);
  m->wdiau = f2_alloc_n(L+1,nx,ny); m->wdiav = f2_alloc_n(L+1,nx,ny);
  m->Fdu = f2_alloc_n(L+1,nx,ny); m->Fdv = f2_alloc_n(L+1,nx,ny);
  m->gprime = f2_alloc_n(L,nx,ny);
  m->huu = f2_alloc_n(L,nx,ny); m->hvv = f2_alloc_n(L,nx,ny);
  {
    F2 * one[] = { &m->hhsw, &m->hhbw, &m->hhs_west, &m->hhs_south, &m->hhb_west,
                   &m->hhb_south, &m->Hc, &m->Hw, &m->Hs, &m->tauxw, &m->tauyw, &m->usqs,
                   &m->vsqs, &m->uabss, &m->usqb, &m->vsqb, &m->uabsb, &m->DDT, &m->DDS,
                   &m->DD4T, &m->DD4S, &m->A2h, &m->A2q, &m->A4h, &m->A4q, &m->UU4,
                   &m->VV4, &m->d2hx, &m->d2hy, &m->dhdx, &m->dhdy, &m->pi, &m->rhs };
    size_t p;
    for (p = 0; p < sizeof(one)/sizeof(one[0]); p ++) f2_alloc(one[p],nx,ny);
  }
  /* defaults of state.c:968-1006 */
  {
    int k;
    for (k = 0; k < L; k ++)
    {
      f2_fill(&m->hRelax[k],1000.0/L);
      f2_fill(&m->eRelax[k],1000.0*k/L);
      f2_fill(&m->uTime[k],-1); f2_fill(&m->vTime[k],-1); f2_fill(&m->eTime[k],-1);
      m->gg[k] = 9.81;
    }
    f2_fill(&m->hTime,-1);
  }
  return m;
}

void orc_destroy (orc_model * m)
{
  int L, lv;
  if (m == NULL) return;
  L = m->L;
  f2_free_n(m->u,L); f2_free_n(m->v,L); f2_free_n(m->h,L);
  for (lv = 0; lv < 3; lv ++) { f2_free_n(m->tu[lv],L); f2_free_n(m->tv[lv],L); f2_free_n(m->th[lv],L); }
  free(m->hhs.d); free(m->hhb.d); free(m->omz.d); free(m->uLid.d); free(m->vLid.d);
  free(m->fbx.d); free(m->fby.d); free(m->hTime.d);
  f2_free_n(m->taux,m->c.tau_nrecs); f2_free_n(m->tauy,m->c.tau_nrecs);
  f2_free_n(m->uRelax,L); f2_free_n(m->vRelax,L); f2_free_n(m->hRelax,L); f2_free_n(m->eRelax,L);
  f2_free_n(m->uTime,L); f2_free_n(m->vTime,L); f2_free_n(m->eTime,L);
  f2_free_n(m->wdia_ff,m->c.wdia_nrecs*(L+1)); f2_free_n(m->nu_u,L); f2_free_n(m->nu_v,L);
  free(m->gg); free(m->geff);
  f2_free_n(m->uw,L); f2_free_n(m->vw,L); f2_free_n(m->hw,L);
  f2_free_n(m->dtu,L); f2_free_n(m->dtv,L); f2_free_n(m->dth,L);
  f2_free_n(m->hwest,L); f2_free_n(m->hsouth,L); f2_free_n(m->hFsw,L); f2_free_n(m->hFss,L);
  f2_free_n(m->hFbw,L); f2_free_n(m->hFbs,L); f2_free_n(m->hhq,L); f2_free_n(m->zeta,L);
  f2_free_n(m->qq,L); f2_free_n(m->al,L); f2_free_n(m->be,L); f2_free_n(m->ga,L);
  f2_free_n(m->de,L); f2_free_n(m->ep,L); f2_free_n(m->ph,L); f2_free_n(m->la,L);
  f2_free_n(m->mu,L); f2_free_n(m->pp,L); f2_free_n(m->KE,L); f2_free_n(m->MM,L);
  f2_free_n(m->eta,L+1); f2_free_n(m->wdia,L+1); f2_free_n(m->wdiau,L+1); f2_free_n(m->wdiav,L+1);
  f2_free_n(m->Fdu,L+1); f2_free_n(m->Fdv,L+1); f2_free_n(m->gprime,L);
  f2_free_n(m->huu,L); f2_free_n(m->hvv,L);
  {
    F2 * one[] = { &m->hhsw, &m->hhbw, &m->hhs_west, &m->hhs_south, &m->hhb_west,
                   &m->hhb_south, &m->Hc, &m->Hw, &m->Hs, &m->tauxw, &m->tauyw, &m->usqs,
                   &m->vsqs, &m->uabss, &m->usqb, &m->vsqb, &m->uabsb, &m->DDT, &m->DDS,
                   &m->DD4T, &m->DD4S, &m->A2h, &m->A2q, &m->A4h, &m->A4q, &m->UU4,
                   &m->VV4, &m->d2hx, &m->d2hy, &m->dhdx, &m->dhdy, &m->pi, &m->rhs };
    size_t p;
    for (p = 0; p < sizeof(one)/sizeof(one[0]); p ++) free(one[p]->d);
  }
  if (m->mg != NULL)
  {
    for (lv = 0; lv < m->Ngrids; lv ++)
    {
      mg_level * l = &m->mg[lv];
      free(l->pi); free(l->pi_temp); free(l->rhs); free(l->Hc); free(l->Hw); free(l->Hs);
      free(l->Ow); free(l->Os); free(l->Osum); free(l->rOsum);
      free(l->wmm); free(l->wmp); free(l->wpm); free(l->wpp);
    }
    free(m->mg);
  }
  free(m->Fmg);
  free(m);
}

/* name -> field lookup for the array API */
static F2 * lookup (orc_model * m, const char * nm, int k, int writing, int * qgrid)
{
  int L = m->L;
  *qgrid = 0;
#define PER(name,arr,n) if (strcmp(nm,name) == 0) return ((k >= 0) && (k < (n))) ? &(arr)[k] : NULL
#define ONE(name,fld) if (strcmp(nm,name) == 0) return &(fld)
  PER("u",m->u,L); PER("v",m->v,L); PER("h",m->h,L);
  ONE("hhs",m->hhs); ONE("hhb",m->hhb);
  if (strcmp(nm,"omegaz") == 0) { *qgrid = 1; return &m->omz; }
  PER("taux",m->taux,m->c.tau_nrecs); PER("tauy",m->tauy,m->c.tau_nrecs);
  ONE("uLid",m->uLid); ONE("vLid",m->vLid); ONE("Fbaro_x",m->fbx); ONE("Fbaro_y",m->fby);
  PER("uRelax",m->uRelax,L); PER("vRelax",m->vRelax,L); PER("hRelax",m->hRelax,L);
  PER("eRelax",m->eRelax,L); PER("uTime",m->uTime,L); PER("vTime",m->vTime,L);
  PER("eTime",m->eTime,L); ONE("hTime",m->hTime);
  PER("wdia_ff",m->wdia_ff,m->c.wdia_nrecs*(L+1));
  PER("nu_u_dia",m->nu_u,L); PER("nu_v_dia",m->nu_v,L);
  if (writing) return NULL;
  PER("dt_u",m->dtu,L); PER("dt_v",m->dtv,L); PER("dt_h",m->dth,L);
  PER("h_west",m->hwest,L); PER("h_south",m->hsouth,L); PER("eta",m->eta,L+1);
  PER("zeta",m->zeta,L); PER("hhq",m->hhq,L); PER("qq",m->qq,L);
  PER("alpha",m->al,L); PER("beta",m->be,L); PER("gamma",m->ga,L); PER("delta",m->de,L);
  PER("epsilon",m->ep,L); PER("phi",m->ph,L); PER("lambda",m->la,L); PER("mu",m->mu,L);
  PER("pp",m->pp,L); PER("KE",m->KE,L); PER("MM",m->MM,L); PER("wdia",m->wdia,L+1);
  ONE("pi",m->pi); ONE("pi_rhs",m->rhs); ONE("Hc",m->Hc); ONE("Hw",m->Hw); ONE("Hs",m->Hs);
  ONE("hhs_west",m->hhs_west); ONE("hhs_south",m->hhs_south);
  ONE("hhb_west",m->hhb_west); ONE("hhb_south",m->hhb_south);
  if ((k >= 0) && (k < 3*L))
  {
    if (strcmp(nm,"tend_u") == 0) return &m->tu[k/L][k%L];
    if (strcmp(nm,"tend_v") == 0) return &m->tv[k/L][k%L];
    if (strcmp(nm,"tend_h") == 0) return &m->th[k/L][k%L];
  }
#undef PER
#undef ONE
  return NULL;
}

int orc_set (orc_model * m, const char * name, int k, const double * src)
{
  int q, i, j;
  F2 * f;
  if (strcmp(name,"gg") == 0)
  {
    memcpy(m->gg,src,(size_t) m->L*sizeof(double));
    return 0;
  }
  f = lookup(m,name,k,1,&q);
  if (f == NULL) return -1;
  if (q)
  {
    /* state.c:207-238: the q line past the last cell exists only on walled sides */
    int qx = m->Nx + (m->c.wall_ew ? 1 : 0), qy = m->Ny + (m->c.wall_ns ? 1 : 0);
    for (j = 0; j < qy; j ++)
      for (i = 0; i < qx; i ++)
        A(f,G+i,G+j) = src[(size_t) j*(m->Nx+1) + i];
    return 0;
  }
  for (j = 0; j < m->Ny; j ++)
    for (i = 0; i < m->Nx; i ++)
      A(f,G+i,G+j) = src[(size_t) j*m->Nx + i];
  return 0;
}

int orc_get (orc_model * m, const char * name, int k, double * dst)
{
  int q, i, j;
  F2 * f;
  if (strcmp(name,"gg") == 0)
  {
    memcpy(dst,m->gg,(size_t) m->L*sizeof(double));
    return 0;
  }
  f = lookup(m,name,k,0,&q);
  if (f == NULL) return -1;
  if (q)
  {
    for (j = 0; j <= m->Ny; j ++)
      for (i = 0; i <= m->Nx; i ++)
        dst[(size_t) j*(m->Nx+1) + i] = A(f,G+i,G+j);
    return 0;
  }
  for (j = 0; j < m->Ny; j ++)
    for (i = 0; i < m->Nx; i ++)
      dst[(size_t) j*m->Nx + i] = A(f,G+i,G+j);
  return 0;
}

/* state.c:1052-1100 */
int orc_init (orc_model * m)
{
  int k, L = m->L;
  state_halos(m,m->u,m->v,m->h);
  xch(m,&m->hhb,K_SCALAR);
  xch(m,&m->hhs,K_SCALAR);
  xch(m,&m->omz,K_Q);
  xch(m,&m->uLid,K_U); xch(m,&m->vLid,K_V);
  xch(m,&m->fbx,K_U); xch(m,&m->fby,K_V);
  for (k = 0; k < m->c.tau_nrecs; k ++) { xch(m,&m->taux[k],K_SCALAR); xch(m,&m->tauy[k],K_SCALAR); }
  for (k = 0; k < m->c.wdia_nrecs*(L+1); k ++) xch(m,&m->wdia_ff[k],K_SCALAR);
  for (k = 0; k < L; k ++)
  {
    xch(m,&m->uRelax[k],K_U); xch(m,&m->vRelax[k],K_V);
    xch(m,&m->hRelax[k],K_SCALAR); xch(m,&m->eRelax[k],K_SCALAR);
    xch(m,&m->uTime[k],K_U); xch(m,&m->vTime[k],K_V); xch(m,&m->eTime[k],K_SCALAR);
    xch(m,&m->nu_u[k],K_U); xch(m,&m->nu_v[k],K_V);
  }
  xch(m,&m->hTime,K_SCALAR);
  m->geff[0] = m->gg[0];
  for (k = 1; k < L; k ++) m->geff[k] = m->geff[k-1] + m->gg[k];
  for (k = 0; k < L; k ++) if (m->gg[k] < 0) return -1;
  return 0;
}
