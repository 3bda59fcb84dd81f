/*
 * CPU oracle: a plain-C restatement of the reference's per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file;
 * only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * use it, and only as the source of expected values.
 *
 * Every routine follows one reference routine (cited file:line) statement for
 * statement in its floating-point arithmetic: the same expressions in the
 * same evaluation order, so that, compiled without contraction
 * (-ffp-contract=off), its results are bit-identical to the reference's own
 * compiled sources.  That identity is pinned by tests/test_oracle_pin.py
 * against oracle/_ref (the reference compiled here) and by the committed
 * fixtures in tests/golden/.
 *
 * Layout: every field is one contiguous array in the reference layout
 * [X_np][Y_m][Z_m] with k fastest (Array.h:7-186), for one x-slab of Nx
 * interior planes i = 3..Nx+2, 3 ghost planes on each side, interior
 * j = 2..Ny+1 (ghost rows 1 and Ny+2) and interior k = 2..Nz+1 (ghost rows 1
 * and Nz+2).  Face arrays keep the reference's shifted indexing: the x-face
 * i+1/2 of cell (i,j,k) is stored at [i][j-1][k-1], the y-face j+1/2 at
 * [i-1][j][k-1], the z-face k+1/2 at [i-1][j-1][k] (Dual_time_stepping.cpp:
 * 810-828).  Two x configurations: periodic (x_open = 0), where the
 * reference's slab decomposition collapses to one slab whose halos wrap
 * around (main.cpp:167-200 and Dual_time_stepping.cpp:942-976 with the single
 * slab as its own neighbour: the reference's interior-rank code paths), and
 * open (x_open = 1), the reference's own inflow/outflow configuration run as
 * a single rank that is both the first and the last (every myid == 0 and
 * myid == nproc-1 branch taken): characteristic X boundaries, one-sided
 * MUSCL stencils at the x ends, no x halo exchange, zero implicit halos,
 * sponge layers of nx_inlet / nx_outlet cells and, optionally, the
 * reference's buoyancy body force.
 *
 * Names below that mirror the reference: jn = "ny" (= Ny+1), kn = "nz"
 * (= Nz+1), ie = gend (= Nx+2), nyy = Ny+2, nzz = Nz+2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>
#include <stdio.h>

#define KG 1.4          /* gamma, prm.h:7 */
#define RG 287.0        /* gas constant, prm.h:8 */
#define CV 717.5        /* Viscous_terms.h:3 */

typedef struct {
  int nx, ny, nz;          /* interior cells */
  double dxi, det, dzt;    /* deltaXI, deltaET, deltaZT */
  double dt, e;            /* deltaT, preconditioning floor e */
  double mu, pr;           /* mu_L, Pr_L */
  double twall_lo, twall_hi;
  double force;            /* uniform x body force replacing Dual_time_stepping.cpp:831 */
  int curved_walls;        /* 1: wall-face momentum flux with the eta_x, eta_z pressure terms */
  int x_open;              /* 1: inflow/outflow x ends (single rank 0 of 1); 0: periodic slab */
  int nx_inlet, nx_outlet; /* sponge layers (Resolution.h), open x only */
  int buoyancy;            /* 1: f = -(rho - 1.1842) 9.81 of Dual_time_stepping.cpp:831 */
} or_params;

typedef struct {
  or_params p;
  int X, Y, Z;             /* X_np, Y_m, Z_m */
  double *U_[5], *U[5], *Uq[5];
  double *J, *m[9];                        /* cell metrics xidx..ztdz */
  double *Jf[3], *mf[3][9];                /* face sets u, v, w */
  double *inF[3][5], *vF[4];
  double *MR[5], *NL[5], *NR[5];
  double *visc[3][4];                      /* face viscous fluxes LL/ML/NL 2..5 */
  double *ML[5], *MRs[5];                  /* MUSCL face states */
  double *res[5];                          /* squared increments of the update */
  double *spg[5];                          /* sponge terms (the reference's Residual arrays) */
  double high;                             /* channel height parameter of prm.h (or_metrics) */
} or_state;

#define IX(s, i, j, k) (((size_t)(i) * (size_t)(s)->Y + (size_t)(j)) * (size_t)(s)->Z + (size_t)(k))
#define MAX(a, b) (((a) > (b)) ? (a) : (b))

static size_t or_n(const or_state *s) { return (size_t)s->X * s->Y * s->Z; }

/* ------------------------------------------------------------------------ */
/* allocation                                                                 */

or_state *or_create(const or_params *p) {
  or_state *s = (or_state *)calloc(1, sizeof(or_state));
  s->p = *p;
  s->X = p->nx + 6; s->Y = p->ny + 4; s->Z = p->nz + 4;
  size_t n = or_n(s);
#define A() ((double *)calloc(n, sizeof(double)))
  for (int v = 0; v < 5; v++) {
    s->U_[v] = A(); s->U[v] = A(); s->Uq[v] = A();
    s->MR[v] = A(); s->NL[v] = A(); s->NR[v] = A();
    s->ML[v] = A(); s->MRs[v] = A(); s->res[v] = A(); s->spg[v] = A();
    for (int d = 0; d < 3; d++) s->inF[d][v] = A();
  }
  for (int v = 0; v < 4; v++) {
    s->vF[v] = A();
    for (int d = 0; d < 3; d++) s->visc[d][v] = A();
  }
  s->J = A();
  for (int v = 0; v < 9; v++) s->m[v] = A();
  for (int d = 0; d < 3; d++) {
    s->Jf[d] = A();
    for (int v = 0; v < 9; v++) s->mf[d][v] = A();
  }
#undef A
  return s;
}

void or_destroy(or_state *s) {
  if (!s) return;
  for (int v = 0; v < 5; v++) {
    free(s->U_[v]); free(s->U[v]); free(s->Uq[v]); free(s->MR[v]); free(s->NL[v]);
    free(s->NR[v]); free(s->ML[v]); free(s->MRs[v]); free(s->res[v]); free(s->spg[v]);
    for (int d = 0; d < 3; d++) free(s->inF[d][v]);
  }
  for (int v = 0; v < 4; v++) {
    free(s->vF[v]);
    for (int d = 0; d < 3; d++) free(s->visc[d][v]);
  }
  free(s->J);
  for (int v = 0; v < 9; v++) free(s->m[v]);
  for (int d = 0; d < 3; d++) { free(s->Jf[d]); for (int v = 0; v < 9; v++) free(s->mf[d][v]); }
  free(s);
}

/* named access for the Python side: returns the array and its length */
double *or_array(or_state *s, const char *name) {
  static const char *mn[9] = {"xidx", "xidy", "xidz", "etdx", "etdy", "etdz", "ztdx", "ztdy", "ztdz"};
  static const char *fs[3] = {"_u", "_v", "_w"};
  char buf[32];
  for (int v = 0; v < 5; v++) {
    snprintf(buf, sizeof buf, "U%d_", v + 1); if (!strcmp(name, buf)) return s->U_[v];
    snprintf(buf, sizeof buf, "U%d", v + 1); if (!strcmp(name, buf)) return s->U[v];
    snprintf(buf, sizeof buf, "U%dq", v + 1); if (!strcmp(name, buf)) return s->Uq[v];
    snprintf(buf, sizeof buf, "MR%d", v + 1); if (!strcmp(name, buf)) return s->MR[v];
    snprintf(buf, sizeof buf, "NL%d", v + 1); if (!strcmp(name, buf)) return s->NL[v];
    snprintf(buf, sizeof buf, "NR%d", v + 1); if (!strcmp(name, buf)) return s->NR[v];
    snprintf(buf, sizeof buf, "inFx%d", v + 1); if (!strcmp(name, buf)) return s->inF[0][v];
    snprintf(buf, sizeof buf, "inFy%d", v + 1); if (!strcmp(name, buf)) return s->inF[1][v];
    snprintf(buf, sizeof buf, "inFz%d", v + 1); if (!strcmp(name, buf)) return s->inF[2][v];
    snprintf(buf, sizeof buf, "Residual%d", v + 1); if (!strcmp(name, buf)) return s->res[v];
    snprintf(buf, sizeof buf, "Sponge%d", v + 1); if (!strcmp(name, buf)) return s->spg[v];
  }
  for (int v = 0; v < 4; v++) {
    snprintf(buf, sizeof buf, "vF%d", v + 2); if (!strcmp(name, buf)) return s->vF[v];
  }
  static const char *vn[3] = {"vflux_x", "vflux_y", "vflux_z"};
  for (int d = 0; d < 3; d++)
    for (int v = 0; v < 4; v++) {
      snprintf(buf, sizeof buf, "%s%d", vn[d], v + 2); if (!strcmp(name, buf)) return s->visc[d][v];
    }
  if (!strcmp(name, "J")) return s->J;
  for (int d = 0; d < 3; d++) {
    snprintf(buf, sizeof buf, "J%s", fs[d]); if (!strcmp(name, buf)) return s->Jf[d];
  }
  for (int v = 0; v < 9; v++) {
    if (!strcmp(name, mn[v])) return s->m[v];
    for (int d = 0; d < 3; d++) {
      snprintf(buf, sizeof buf, "%s%s", mn[v], fs[d]); if (!strcmp(name, buf)) return s->mf[d][v];
    }
  }
  return NULL;
}

void or_set_force(or_state *s, double f) { s->p.force = f; }

/* ------------------------------------------------------------------------ */
/* metrics: Jacobian.cpp:61-243, Jacobian_u.cpp:59-101, Jacobian_v.cpp:79-151, */
/* Jacobian_w.cpp:61-106 for the interior slab (all x planes 0..Nx+5)         */

void or_metrics(or_state *s, double high, double gam) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1, nyy = jn + 1, nzz = kn + 1;
  const int open = s->p.x_open;
  double **m = s->m;
  s->high = high;
  /* cell metrics, Jacobian.cpp:53-107 (interior rank: planes 0..gend+3;
   * first and last rank: 3..gend) */
  for (int i = open ? 3 : 0; i <= (open ? ie : ie + 3); i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        double etdy, ydet;
        /* Jacobian.cpp:77 evaluates temp2 with 1/cosh (integer one) */
        double temp = (0.5 * high) * (1 - 1. / tanh(gam) * tanh(gam * (1 - 2 * (j - 1.5) * s->p.det)));
        double temp1 = (1 - temp / (0.5 * high)) * tanh(gam);
        double temp2 = 1 / cosh(gam * (1 - 2 * (j - 1.5) * s->p.det));
        etdy = tanh(gam) / (2 * (0.5 * high) * gam * (1 - temp1 * temp1));
        ydet = high * gam * 1. / tanh(gam) * temp2 * temp2;
        m[0][c] = 1; m[1][c] = 0; m[2][c] = 0;
        m[3][c] = 0; m[4][c] = etdy; m[5][c] = 0;
        m[6][c] = 0; m[7][c] = 0; m[8][c] = 1;
        s->J[c] = 1. / (1 * ydet * 1);
      }
  /* x-end planes of the first and last rank, Jacobian.cpp:110-157: copies
   * of the neighbouring interior plane over j, k = 1..Ny+2 / Nz+2 (its ghost
   * rows are not set yet), where ztdx is copied three times and ztdy, ztdz
   * of the end plane stay zero */
  if (open)
    for (int side = 0; side < 2; side++) {
      int ig = side ? ie + 1 : 2, is = side ? ie : 3;
      for (int j = 1; j <= nyy; j++)
        for (int k = 1; k <= nzz; k++) {
          size_t g = IX(s, ig, j, k), c = IX(s, is, j, k);
          for (int v = 0; v < 7; v++) m[v][g] = m[v][c];
          s->J[g] = s->J[c];
        }
    }
  /* y ghost rows, Jacobian.cpp:159-200 (planes 0..gend+3, or 2..gend+1 on
   * an open slab), with the copy typos that leave ztdy = ztdz = ztdx of the
   * neighbour (= 0) in the ghost rows */
  for (int i = open ? 2 : 0; i <= (open ? ie + 1 : ie + 3); i++)
    for (int k = 2; k <= kn; k++) {
      for (int side = 0; side < 2; side++) {
        int jg = side ? nyy : 1, js = side ? jn : 2;
        size_t g = IX(s, i, jg, k), c = IX(s, i, js, k);
        m[0][g] = m[0][c]; m[1][g] = m[1][c]; m[2][g] = m[2][c];
        m[3][g] = m[3][c]; m[4][g] = m[4][c]; m[5][g] = m[5][c];
        m[6][g] = m[6][c]; m[7][g] = m[6][c]; m[8][g] = m[6][c];
      }
      s->J[IX(s, i, 1, k)] = s->J[IX(s, i, 2, k)];
      s->J[IX(s, i, nyy, k)] = s->J[IX(s, i, jn, k)];
    }
  /* z ghost rows, Jacobian.cpp:203-243, same typos and plane range */
  for (int i = open ? 2 : 0; i <= (open ? ie + 1 : ie + 3); i++)
    for (int j = 1; j <= nyy; j++) {
      for (int side = 0; side < 2; side++) {
        int kg = side ? nzz : 1, ks = side ? kn : 2;
        size_t g = IX(s, i, j, kg), c = IX(s, i, j, ks);
        m[0][g] = m[0][c]; m[1][g] = m[1][c]; m[2][g] = m[2][c];
        m[3][g] = m[3][c]; m[4][g] = m[4][c]; m[5][g] = m[5][c];
        m[6][g] = m[6][c]; m[7][g] = m[6][c]; m[8][g] = m[6][c];
      }
      s->J[IX(s, i, j, 1)] = s->J[IX(s, i, j, 2)];
      s->J[IX(s, i, j, nzz)] = s->J[IX(s, i, j, kn)];
    }
  /* face sets: u = x-faces (Jacobian_u.cpp:59-101, eta at j-0.5),
   * v = y-faces (Jacobian_v.cpp:79-151, eta at j-1.0, then wall rows
   * replaced by cell values), w = z-faces (Jacobian_w.cpp:61-106) */
  struct { int i0, i1, j0, j1, k0, k1; double off; } fr[3] = {
    {2, ie, 1, jn - 1, 1, kn - 1, 0.5},
    {2, ie - 1, 1, jn, 1, kn - 1, 1.0},
    {2, ie - 1, 1, jn - 1, 1, kn, 0.5},
  };
  for (int d = 0; d < 3; d++)
    for (int i = fr[d].i0; i <= fr[d].i1; i++)
      for (int j = fr[d].j0; j <= fr[d].j1; j++)
        for (int k = fr[d].k0; k <= fr[d].k1; k++) {
          size_t c = IX(s, i, j, k);
          double temp = (0.5 * high) * (1 - 1. / tanh(gam) * tanh(gam * (1 - 2 * (j - fr[d].off) * s->p.det)));
          double temp1 = (1 - temp / (0.5 * high)) * tanh(gam);
          double temp2 = (d == 1) ? 1 / cosh(gam * (1 - 2 * (j - fr[d].off) * s->p.det))
                                  : 1. / cosh(gam * (1 - 2 * (j - fr[d].off) * s->p.det));
          double **mf = s->mf[d];
          mf[0][c] = 1; mf[1][c] = 0; mf[2][c] = 0;
          mf[3][c] = 0; mf[4][c] = tanh(gam) / (2 * (0.5 * high) * gam * (1 - temp1 * temp1)); mf[5][c] = 0;
          mf[6][c] = 0; mf[7][c] = 0; mf[8][c] = 1;
          double ydet = high * gam * 1. / tanh(gam) * temp2 * temp2;
          s->Jf[d][c] = 1. / (1 * ydet * 1);
        }
  /* Jacobian_v.cpp:134-151: wall faces take the ghost-cell metric */
  for (int i = 2; i <= ie - 1; i++)
    for (int k = 1; k < kn; k++) {
      size_t f1 = IX(s, i, 1, k), fn = IX(s, i, jn, k);
      s->mf[1][3][f1] = m[3][IX(s, i, 1, k)];
      s->mf[1][4][f1] = m[4][IX(s, i, 1, k)];
      s->mf[1][5][f1] = m[5][IX(s, i, 1, k)];
      s->mf[1][3][fn] = m[3][IX(s, i, nyy, k)];
      s->mf[1][4][fn] = m[4][IX(s, i, nyy, k)];
      s->mf[1][5][fn] = m[5][IX(s, i, nyy, k)];
      s->Jf[1][fn] = s->J[IX(s, i, nyy, k)];
      s->Jf[1][f1] = s->J[IX(s, i, 1, k)];
    }
}

/* ------------------------------------------------------------------------ */
/* initial condition: Initial_condition.cpp:56-97 then :187-221 (restart     */
/* read, switch_initial = 1) and main.cpp:127-141.  q_n, q_nm1: (5,Nx,Ny,Nz)  */
/* physical conserved values, k fastest.                                      */

void or_initial(or_state *s, const double *q_n, const double *q_nm1) {
  const int ie = s->p.nx + 2, Ny = s->p.ny, Nz = s->p.nz;
  const int nyyy = Ny + 3, nzzz = Nz + 3;
  /* the quiescent field of :56-97 also fills the x-end planes 2 and gend+1
   * of the first and last rank */
  const int open = s->p.x_open;
  for (int i = open ? 2 : 3; i <= (open ? ie + 1 : ie); i++)
    for (int j = 0; j <= nyyy; j++)
      for (int k = 0; k <= nzzz; k++) {
        size_t c = IX(s, i, j, k);
        double T = 298.0592, U = 0, V = 0, W = 0;
        double VV = U * U + V * V + W * W;
        double P = 101300;
        double rho = P / T / RG;
        double q[5] = {rho / s->J[c], rho * U / s->J[c], rho * V / s->J[c], rho * W / s->J[c],
                       (P / (KG - 1) + 0.5 * rho * VV) / s->J[c]};
        for (int v = 0; v < 5; v++) { s->U[v][c] = q[v]; s->Uq[v][c] = q[v]; s->U_[v][c] = q[v]; }
      }
  size_t nint = (size_t)s->p.nx * Ny * Nz;
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= Ny + 1; j++)
      for (int k = 2; k <= Nz + 1; k++) {
        size_t c = IX(s, i, j, k);
        size_t ii = ((size_t)(i - 3) * Ny + (j - 2)) * Nz + (k - 2);
        for (int v = 0; v < 5; v++) {
          s->U[v][c] = q_n[v * nint + ii] / s->J[c];
          s->Uq[v][c] = q_nm1[v * nint + ii] / s->J[c];
          s->U_[v][c] = s->U[v][c];
        }
      }
}

/* ------------------------------------------------------------------------ */
/* boundary conditions                                                       */

/* periodic x halo of Q/J, main.cpp:167-200 with the slab as its own neighbour */
void or_halo_x(or_state *s) {
  const int ie = s->p.nx + 2;
  if (s->p.x_open) return;   /* both neighbours are MPI_PROC_NULL */
  size_t plane = (size_t)s->Y * s->Z;
  for (int v = 0; v < 5; v++) {
    memmove(s->U_[v] + (size_t)(ie + 1) * plane, s->U_[v] + (size_t)3 * plane, 3 * plane * sizeof(double));
    memmove(s->U_[v] + 0, s->U_[v] + (size_t)(ie - 2) * plane, 3 * plane * sizeof(double));
  }
}

/* walls, Y_boundary_condition.cpp:94-182: zero-gradient copy, then
 * no-slip isothermal reflection inside the heated section (global plane
 * i + gstart in (nx_inlet + 2, X_out - nx_outlet + 3), :114; every plane
 * without sponge layers; the slab is planes 1..Nx of the x extent here) */
void or_bc_y(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1, nyy = jn + 1;
  double **q = s->U_;
  const double *J = s->J;
  for (int i = 3; i <= ie; i++) {
    for (int k = 2; k <= kn; k++)
      for (int v = 0; v < 5; v++) {
        q[v][IX(s, i, 1, k)] = q[v][IX(s, i, 2, k)];
        q[v][IX(s, i, nyy, k)] = q[v][IX(s, i, jn, k)];
      }
    if (!(i > s->p.nx_inlet + 2 && i < s->p.nx - s->p.nx_outlet + 3)) continue;
    for (int k = 2; k <= kn; k++) {
      for (int side = 0; side < 2; side++) {
        int js = side ? jn : 2, jg = side ? nyy : 1;
        size_t c = IX(s, i, js, k), g = IX(s, i, jg, k);
        double rho = q[0][c] * J[c];
        double U = q[1][c] / q[0][c];
        double V = q[2][c] / q[0][c];
        double W = q[3][c] / q[0][c];
        double VV = U * U + V * V + W * W;
        double P = (q[4][c] * J[c] - 0.5 * rho * VV) * (KG - 1);
        double T = side ? s->p.twall_hi : s->p.twall_lo;
        rho = P / RG / T;
        q[0][g] = rho / J[g];
        q[1][g] = -rho * U / J[g];
        q[2][g] = -rho * V / J[g];
        q[3][g] = -rho * W / J[g];
        q[4][g] = (P / (KG - 1) + 0.5 * rho * VV) / J[g];
      }
    }
  }
}

/* characteristic inflow / outflow ghost planes of an open slab,
 * X_boundary_condition.cpp:73-338: the ghost cell of each interior row takes
 * one pseudo-time step of deltaT/200 with M (Gamma + 3 dtau/(2 dt) M)^-1
 * applied to the wave amplitudes (outgoing from the one-sided x
 * differences, incoming zero) plus the BDF2 time derivative.  side 0:
 * inlet plane 2 against plane 3; side 1: outlet plane gend+1 against gend. */
static void bc_x_side(or_state *s, int side) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  const double K = KG, deltaT = s->p.dt, deltaTau = deltaT / 200., e = s->p.e, dXI = s->p.dxi;
  const int ig = side ? ie + 1 : 2, ii = side ? ie : 3;
  double **q = s->U_, **u = s->U, **uq = s->Uq;
  const double *Jc = s->J;
  for (int j = 2; j <= jn; j++)
    for (int k = 2; k <= kn; k++) {
      size_t c = IX(s, ii, j, k), g = IX(s, ig, j, k);
      /* the interior neighbour */
      double rho_ = q[0][c] * Jc[c];
      double U_ = q[1][c] / q[0][c];
      double V_ = q[2][c] / q[0][c];
      double W_ = q[3][c] / q[0][c];
      double VV_ = U_ * U_ + V_ * V_ + W_ * W_;
      double P_ = (q[4][c] * Jc[c] - 0.5 * rho_ * VV_) * (K - 1);
      double T_ = P_ / rho_;
      (void)VV_;
      /* the ghost cell */
      double rho = q[0][g] * Jc[g];
      double U = q[1][g] / q[0][g];
      double V = q[2][g] / q[0][g];
      double W = q[3][g] / q[0][g];
      double VV = U * U + V * V + W * W;
      double P = (q[4][g] * Jc[g] - 0.5 * rho * VV) * (K - 1);
      double C = sqrt(K * P / rho);
      double T = P / rho;
      double H = 0.5 * VV + C * C / (K - 1);
      double beta = MAX(VV / C / C, e);
      double temp = K * T * (2 * deltaT + 3 * deltaTau) * (2 * deltaT + 3 * beta * deltaTau);
      double temp2 = (K - 1) * (beta - 1) * deltaT * deltaT;
      double temp3 = H - H * K - VV + K * (T + VV);
      double d[5][5];
      d[0][0] = (2 * deltaT * (-2 * (-(K - 1) * (H - VV) - temp3 * beta) * deltaT + 3 * K * T * beta * deltaTau)) / temp;
      d[0][1] = (-4 * U * temp2) / temp;
      d[0][2] = (-4 * V * temp2) / temp;
      d[0][3] = (-4 * W * temp2) / temp;
      d[0][4] = (4 * temp2) / temp;
      d[1][0] = (4 * U * temp3 * (beta - 1) * deltaT * deltaT) / temp;
      d[1][1] = (2 * deltaT * (2 * K * (T - U * U * (beta - 1)) * deltaT + 2 * U * U * (beta - 1) * deltaT + 3 * K * T * beta * deltaTau)) / temp;
      d[1][2] = (-4 * U * V * temp2) / temp;
      d[1][3] = (-4 * U * W * temp2) / temp;
      d[1][4] = (4 * U * temp2) / temp;
      d[2][0] = (4 * V * temp3 * (beta - 1) * deltaT * deltaT) / temp;
      d[2][1] = (-4 * U * V * temp2) / temp;
      d[2][2] = (2 * deltaT * (2 * K * (T - V * V * (beta - 1)) * deltaT + 2 * V * V * (beta - 1) * deltaT + 3 * K * T * beta * deltaTau)) / temp;
      d[2][3] = (-4 * V * W * temp2) / temp;
      d[2][4] = (4 * V * temp2) / temp;
      d[3][0] = (4 * W * temp3 * (beta - 1) * deltaT * deltaT) / temp;
      d[3][1] = (-4 * U * W * temp2) / temp;
      d[3][2] = (-4 * V * W * temp2) / temp;
      d[3][3] = (2 * deltaT * (2 * K * (T - W * W * (beta - 1)) * deltaT + 2 * W * W * (beta - 1) * deltaT + 3 * K * T * beta * deltaTau)) / temp;
      d[3][4] = (4 * W * temp2) / temp;
      d[4][0] = (4 * H * temp3 * (beta - 1) * deltaT * deltaT) / temp;
      d[4][1] = (-4 * H * U * temp2) / temp;
      d[4][2] = (-4 * H * V * temp2) / temp;
      d[4][3] = (-4 * H * W * temp2) / temp;
      d[4][4] = (2 * deltaT * (2 * H * (K - 1) * (beta - 1) * deltaT + K * T * (2 * deltaT + 3 * beta * deltaTau))) / temp;
      double U_p = 0.5 * (beta + 1) * U;
      double C_p = 0.5 * sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * C * C);
      double dp_dx, du_dx, dv_dx, dw_dx, dT_dx, L1, L2, L3, L4, L5;
      if (!side) {   /* :151-187: L5 leaves through the inlet, L4 from it */
        dp_dx = (P_ - P) / dXI;
        du_dx = (U_ - U) / dXI;
        dv_dx = (V_ - V) / dXI;
        dw_dx = (W_ - W) / dXI;
        dT_dx = (T_ - T) / dXI;
        L5 = (U_p - C_p) * (dp_dx - rho * (U_p + C_p - U) * du_dx);
        L4 = L5 * (U_p - C_p - U) / (U_p + C_p - U);
        if (U <= 0) {
          L1 = U * (dT_dx + 1.0 / rho * dp_dx * (1 - K) / K);
          L2 = U * dw_dx;
          L3 = -U * dv_dx;
        } else {
          L1 = L2 = L3 = 0;
        }
      } else {       /* :292-327 */
        dp_dx = (P - P_) / dXI;
        du_dx = (U - U_) / dXI;
        dv_dx = (V - V_) / dXI;
        dw_dx = (W - W_) / dXI;
        dT_dx = (T - T_) / dXI;
        L4 = (U_p + C_p) * (dp_dx - rho * (U_p - C_p - U) * du_dx);
        L5 = L4 * (U_p + C_p - U) / (U_p - C_p - U);
        if (U > 0) {
          L1 = U * (dT_dx + 1.0 / rho * dp_dx * (1 - K) / K);
          L2 = U * dw_dx;
          L3 = -U * dv_dx;
        } else {
          L1 = L2 = L3 = 0;
        }
      }
      double KAL[5];
      KAL[0] = 0.5 / (C_p) * (L4 * (U_p + C_p - U) - L5 * (U_p - C_p - U));
      KAL[1] = 0.5 / (rho * C_p) * (L4 - L5);
      KAL[2] = -L3;
      KAL[3] = L2;
      KAL[4] = L1 + 1. / rho * (K - 1) / K * KAL[0];
      for (int v = 0; v < 5; v++)
        KAL[v] = KAL[v] / Jc[g] + (3 * q[v][g] - 4 * u[v][g] + uq[v][g]) / (2 * deltaT);
      for (int v = 0; v < 5; v++)
        q[v][g] = q[v][g] - deltaTau * (d[v][0] * KAL[0] + d[v][1] * KAL[1] + d[v][2] * KAL[2] + d[v][3] * KAL[3] +
                                        d[v][4] * KAL[4]);
    }
}

void or_bc_x(or_state *s) {
  if (!s->p.x_open) return;   /* interior rank: no-op */
  bc_x_side(s, 0);
  bc_x_side(s, 1);
}

/* periodic z ghosts, Z_boundary_condition.cpp:39-66 (all planes, all rows) */
void or_bc_z(or_state *s) {
  const int ie = s->p.nx + 2, kn = s->p.nz + 1, nzz = kn + 1, nyyy = s->p.ny + 3;
  const int open = s->p.x_open;   /* :40-44: planes 2..gend+1 on an open slab */
  for (int i = open ? 2 : 0; i <= (open ? ie + 1 : ie + 3); i++)
    for (int j = 0; j <= nyyy; j++)
      for (int v = 0; v < 5; v++) {
        s->U_[v][IX(s, i, j, 1)] = s->U_[v][IX(s, i, j, kn)];
        s->U_[v][IX(s, i, j, nzz)] = s->U_[v][IX(s, i, j, 2)];
      }
}

/* ------------------------------------------------------------------------ */
/* MUSCL reconstruction of Q/J weighted by 1/J (Flux_X.cpp:106-126)          */

static inline double m5L(const double *u, const double *J, size_t a, size_t b, size_t c, size_t d, size_t e) {
  double t = 1. / (2 / J[a] - 13 / J[b] + 47 / J[c] + 27 / J[d] - 3 / J[e]);
  return t * (2 * u[a] - 13 * u[b] + 47 * u[c] + 27 * u[d] - 3 * u[e]);
}
static inline double m5R(const double *u, const double *J, size_t a, size_t b, size_t c, size_t d, size_t e) {
  double t = 1. / (-3 / J[a] + 27 / J[b] + 47 / J[c] - 13 / J[d] + 2 / J[e]);
  return t * (-3 * u[a] + 27 * u[b] + 47 * u[c] - 13 * u[d] + 2 * u[e]);
}
static inline double m3L(const double *u, const double *J, size_t a, size_t b, size_t c) {
  double t = 1. / (-1 / J[a] + 5 / J[b] + 2 / J[c]);
  return t * (-u[a] + 5 * u[b] + 2 * u[c]);
}
static inline double m3R(const double *u, const double *J, size_t a, size_t b, size_t c) {
  double t = 1. / (2 / J[a] + 5 / J[b] - 1 / J[c]);
  return t * (2 * u[a] + 5 * u[b] - u[c]);
}
static inline double m2(const double *u, const double *J, size_t a, size_t b) {
  double t = 1. / (1 / J[a] + 1 / J[b]);
  return t * (u[a] + u[b]);
}

/* preconditioned Roe flux through one face, Flux_X.cpp:229-350 (and the
 * same statements in Flux_Y.cpp:291-396, Flux_Z.cpp:250-354).  L, R: left
 * and right MUSCL states (Q/J weighted); mx,my,mz: face metric; Jf: face J. */
static void roe_face(const double L[5], const double Rr[5], double mx, double my, double mz,
                     double Jf, double e, double F[5], double *Fav3_out, double *pp_out) {
  double insqr = 1.0 / sqrt(mx * mx + my * my + mz * mz);
  double NX = mx * insqr, NY = my * insqr, NZ = mz * insqr;
  double _rho = L[0], _u = L[1] / _rho, _v = L[2] / _rho, _w = L[3] / _rho;
  double iU = mx * _u + my * _v + mz * _w;
  double _VV = _u * _u + _v * _v + _w * _w;
  double iP = (L[4] - 0.5 * _rho * _VV) * (KG - 1);
  double iC = KG * iP / _rho;
  double _H = 0.5 * _VV + iC / (KG - 1);
  double rho_ = Rr[0], u_ = Rr[1] / rho_, v_ = Rr[2] / rho_, w_ = Rr[3] / rho_;
  double U_ = mx * u_ + my * v_ + mz * w_;
  double VV_ = u_ * u_ + v_ * v_ + w_ * w_;
  double P_ = (Rr[4] - 0.5 * rho_ * VV_) * (KG - 1);
  double C_ = KG * P_ / rho_;
  double H_ = 0.5 * VV_ + C_ / (KG - 1);
  double temp5 = sqrt(_rho), temp6 = sqrt(rho_);
  double temp4 = temp5 + temp6;
  double rho = sqrt(_rho * rho_);
  double u = (temp5 * _u + temp6 * u_) / temp4;
  double v = (temp5 * _v + temp6 * v_) / temp4;
  double w = (temp5 * _w + temp6 * w_) / temp4;
  double U = (temp5 * iU + temp6 * U_) / temp4;
  double VV = u * u + v * v + w * w;
  double H = (temp5 * _H + temp6 * H_) / temp4;
  double C = (H - 0.5 * VV) * (KG - 1);
  double dU1 = rho_ - _rho;
  double dU2 = rho_ * u_ - _rho * _u;
  double dU3 = rho_ * v_ - _rho * _v;
  double dU4 = rho_ * w_ - _rho * _w;
  double dU5 = (P_ / (KG - 1) + 0.5 * rho_ * VV_) - (iP / (KG - 1) + 0.5 * _rho * _VV);
  double beta = MAX(VV / C, e);
  double temp = 0.5 * (1 + beta) * U * insqr;
  double S = 0.5 * sqrt(4 * beta * C + U * insqr * U * insqr * (1 - beta) * (1 - beta));
  double theda_p = VV / C;
  double U_p = 0.5 * (1 + theda_p) * U * insqr;
  double C_p = 0.5 * sqrt(4 * C * theda_p + U * insqr * U * insqr * (1 - theda_p) * (1 - theda_p));
  double temp1 = (P_ - iP) / rho / beta / C;
  double temp2 = U_p / S * (U_ - iU) * insqr;
  double temp3 = 0.5 * (1 - beta) * U * insqr * temp / S;
  temp4 = 0.5 * (1 - theda_p) * U * insqr * U_p / S;
  double deltaU = (S - temp3 - beta * fabs(U) * insqr) * temp1 + temp2;
  double deltaP = U_p / S * (P_ - iP) + (C_p - fabs(U) * insqr + temp4) * rho * (U_ - iU) * insqr;
  double Fav1 = fabs(U * insqr) * dU1 + deltaU * rho;
  double Fav2 = fabs(U * insqr) * dU2 + deltaU * rho * u + deltaP * NX;
  double Fav3 = fabs(U * insqr) * dU3 + deltaU * rho * v + deltaP * NY;
  double Fav4 = fabs(U * insqr) * dU4 + deltaU * rho * w + deltaP * NZ;
  double Fav5 = fabs(U * insqr) * dU5 + deltaU * rho * H + deltaP * U * insqr;
  F[0] = 0.5 * ((_rho * iU + rho_ * U_) - Fav1 / insqr) / Jf;
  F[1] = 0.5 * ((_rho * _u * iU + rho_ * u_ * U_ + mx * (iP + P_)) - Fav2 / insqr) / Jf;
  F[2] = 0.5 * ((_rho * _v * iU + rho_ * v_ * U_ + my * (iP + P_)) - Fav3 / insqr) / Jf;
  F[3] = 0.5 * ((_rho * _w * iU + rho_ * w_ * U_ + mz * (iP + P_)) - Fav4 / insqr) / Jf;
  F[4] = 0.5 * ((iU * (3.5 * iP + 0.5 * _rho * _VV) + U_ * (3.5 * P_ + 0.5 * rho_ * VV_)) - Fav5 / insqr) / Jf;
  if (Fav3_out) *Fav3_out = Fav3;
  if (pp_out) *pp_out = iP + P_;
}

/* x-direction inviscid flux, Flux_X.cpp:96-357.  Interior rank: 5-point
 * states for i = 2..gend+1.  Open slab: 5-point for i = 4..gend-1 and the
 * first / last rank's reduced stencils of :139-216 (2-point states on the
 * end faces, 3-point on the next ones) */
void or_flux_x(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  const size_t di = (size_t)s->Y * s->Z;
  const int open = s->p.x_open;
  for (int i = open ? 4 : 2; i <= (open ? ie - 1 : ie + 1); i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        size_t fl = IX(s, i, j - 1, k - 1), fr = IX(s, i - 1, j - 1, k - 1);
        for (int v = 0; v < 5; v++) {
          s->ML[v][fl] = m5L(s->U_[v], s->J, c - 2 * di, c - di, c, c + di, c + 2 * di);
          s->MRs[v][fr] = m5R(s->U_[v], s->J, c - 2 * di, c - di, c, c + di, c + 2 * di);
        }
      }
  if (open)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t a = IX(s, 2, j, k), b = a + di, c = b + di;          /* planes 2, 3, 4 */
        size_t y = IX(s, ie - 1, j, k), z = y + di, w = z + di;    /* planes ie-1, ie, ie+1 */
        for (int v = 0; v < 5; v++) {
          const double *u = s->U_[v];
          s->ML[v][IX(s, 2, j - 1, k - 1)] = m2(u, s->J, a, b);
          s->ML[v][IX(s, 3, j - 1, k - 1)] = m3L(u, s->J, a, b, c);
          s->MRs[v][IX(s, 2, j - 1, k - 1)] = m3R(u, s->J, a, b, c);
          s->ML[v][IX(s, ie, j - 1, k - 1)] = m3L(u, s->J, y, z, w);
          s->MRs[v][IX(s, ie - 1, j - 1, k - 1)] = m3R(u, s->J, y, z, w);
          s->MRs[v][IX(s, ie, j - 1, k - 1)] = m2(u, s->J, z, w);
        }
      }
  double **mf = s->mf[0];
  for (int i = 2; i <= ie; i++)
    for (int j = 1; j < jn; j++)
      for (int k = 1; k < kn; k++) {
        size_t f = IX(s, i, j, k);
        double L[5], R[5], F[5];
        for (int v = 0; v < 5; v++) { L[v] = s->ML[v][f]; R[v] = s->MRs[v][f]; }
        roe_face(L, R, mf[0][f], mf[1][f], mf[2][f], s->Jf[0][f], s->p.e, F, NULL, NULL);
        for (int v = 0; v < 5; v++) s->inF[0][v][f] = F[v];
      }
}

/* y-direction inviscid flux with the reduced stencils next to the walls and
 * the wall-face flux, Flux_Y.cpp:94-413 on an interior rank */
void or_flux_y(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  const size_t dj = (size_t)s->Z;
  for (int i = 3; i <= ie; i++)
    for (int v = 0; v < 5; v++) {
      const double *u = s->U_[v], *J = s->J;
      double *ML = s->ML[v], *MR = s->MRs[v];
      for (int j = 4; j <= jn - 2; j++)
        for (int k = 2; k <= kn; k++) {
          size_t c = IX(s, i, j, k);
          ML[IX(s, i - 1, j, k - 1)] = m5L(u, J, c - 2 * dj, c - dj, c, c + dj, c + 2 * dj);
          MR[IX(s, i - 1, j - 1, k - 1)] = m5R(u, J, c - 2 * dj, c - dj, c, c + dj, c + 2 * dj);
        }
      for (int k = 2; k <= kn; k++) {
        size_t c1 = IX(s, i, 1, k), c2 = IX(s, i, 2, k), c3 = IX(s, i, 3, k), c4 = IX(s, i, 4, k);
        size_t cn = IX(s, i, jn, k), cn1 = IX(s, i, jn - 1, k), cn2 = IX(s, i, jn - 2, k), cg = IX(s, i, jn + 1, k);
        ML[IX(s, i - 1, 1, k - 1)] = m2(u, J, c1, c2);
        ML[IX(s, i - 1, 2, k - 1)] = m2(u, J, c2, c3);
        MR[IX(s, i - 1, 1, k - 1)] = m2(u, J, c2, c3);
        ML[IX(s, i - 1, 3, k - 1)] = m3L(u, J, c2, c3, c4);
        MR[IX(s, i - 1, 2, k - 1)] = m3R(u, J, c2, c3, c4);
        ML[IX(s, i - 1, jn - 1, k - 1)] = m3L(u, J, cn2, cn1, cn);
        MR[IX(s, i - 1, jn - 2, k - 1)] = m3R(u, J, cn2, cn1, cn);
        ML[IX(s, i - 1, jn, k - 1)] = m2(u, J, cn, cn1);
        MR[IX(s, i - 1, jn - 1, k - 1)] = m2(u, J, cn, cn1);
        MR[IX(s, i - 1, jn, k - 1)] = m2(u, J, cn, cg);
      }
    }
  double **mf = s->mf[1];
  for (int i = 2; i <= ie - 1; i++)
    for (int j = 1; j <= jn; j++)
      for (int k = 1; k < kn; k++) {
        size_t f = IX(s, i, j, k);
        double L[5], R[5], F[5], Fav3, pp;
        for (int v = 0; v < 5; v++) { L[v] = s->ML[v][f]; R[v] = s->MRs[v][f]; }
        roe_face(L, R, mf[3][f], mf[4][f], mf[5][f], s->Jf[1][f], s->p.e, F, &Fav3, &pp);
        if (j == 1 || j == jn) {
          F[0] = 0; F[1] = 0; F[3] = 0; F[4] = 0;
          F[2] = 0.5 * (mf[4][f] * pp - 1. * Fav3) / s->Jf[1][f];
          /* Flux_Y.cpp:400-408 assumes flat walls (eta_x = eta_z = 0): a
           * curved wall also carries the x and z pressure force */
          if (s->p.curved_walls) {
            F[1] = 0.5 * (mf[3][f] * pp) / s->Jf[1][f];
            F[3] = 0.5 * (mf[5][f] * pp) / s->Jf[1][f];
          }
        }
        for (int v = 0; v < 5; v++) s->inF[1][v][f] = F[v];
      }
}

/* z-direction inviscid flux with the one-sided stencils next to the z ghost
 * rows, Flux_Z.cpp:91-359 on an interior rank */
void or_flux_z(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  for (int i = 3; i <= ie; i++)
    for (int v = 0; v < 5; v++) {
      const double *u = s->U_[v], *J = s->J;
      double *ML = s->ML[v], *MR = s->MRs[v];
      for (int j = 2; j <= jn; j++) {
        for (int k = 3; k <= kn - 1; k++) {
          size_t c = IX(s, i, j, k);
          ML[IX(s, i - 1, j - 1, k)] = m5L(u, J, c - 2, c - 1, c, c + 1, c + 2);
          MR[IX(s, i - 1, j - 1, k - 1)] = m5R(u, J, c - 2, c - 1, c, c + 1, c + 2);
        }
      }
      for (int j = 2; j <= jn; j++) {
        size_t c1 = IX(s, i, j, 1);
        ML[IX(s, i - 1, j - 1, 1)] = m2(u, J, c1, c1 + 1);
        size_t c = IX(s, i, j, 2);
        ML[IX(s, i - 1, j - 1, 2)] = m3L(u, J, c - 1, c, c + 1);
        MR[IX(s, i - 1, j - 1, 1)] = m3R(u, J, c - 1, c, c + 1);
        c = IX(s, i, j, kn);
        ML[IX(s, i - 1, j - 1, kn)] = m3L(u, J, c - 1, c, c + 1);
        MR[IX(s, i - 1, j - 1, kn - 1)] = m3R(u, J, c - 1, c, c + 1);
        MR[IX(s, i - 1, j - 1, kn)] = m2(u, J, c, c + 1);
      }
    }
  double **mf = s->mf[2];
  for (int i = 2; i <= ie - 1; i++)
    for (int j = 1; j < jn; j++)
      for (int k = 1; k <= kn; k++) {
        size_t f = IX(s, i, j, k);
        double L[5], R[5], F[5];
        for (int v = 0; v < 5; v++) { L[v] = s->ML[v][f]; R[v] = s->MRs[v][f]; }
        roe_face(L, R, mf[6][f], mf[7][f], mf[8][f], s->Jf[2][f], s->p.e, F, NULL, NULL);
        for (int v = 0; v < 5; v++) s->inF[2][v][f] = F[v];
      }
}

/* ------------------------------------------------------------------------ */
/* viscous terms, Viscous_terms.cpp:205-904                                  */

typedef struct { double U, V, W, T; } vprim;

static inline vprim vp_at(const or_state *s, size_t c) {
  vprim r;
  double rho = s->U_[0][c];
  r.U = s->U_[1][c] / rho;
  r.V = s->U_[2][c] / rho;
  r.W = s->U_[3][c] / rho;
  double P = (s->U_[4][c] - 0.5 * rho * (r.U * r.U + r.V * r.V + r.W * r.W)) * (KG - 1) * s->J[c];
  r.T = P / (rho * RG) / s->J[c];
  return r;
}

typedef struct { double a[8], b[8], c[8], d[11], e[11], f[11]; } mcoef;

/* metric products a1..f10 of Viscous_terms.cpp:464-519 */
static void metric_products(const double *x, mcoef *q) {
  double xix = x[0], xiy = x[1], xiz = x[2], etx = x[3], ety = x[4], etz = x[5], ztx = x[6], zty = x[7], ztz = x[8];
  q->a[1] = (4. / 3) * xix * xix + xiy * xiy + xiz * xiz;
  q->a[2] = xix * xix + (4. / 3) * xiy * xiy + xiz * xiz;
  q->a[3] = xix * xix + xiy * xiy + (4. / 3) * xiz * xiz;
  q->a[4] = xix * xix + xiy * xiy + xiz * xiz;
  q->a[5] = (1. / 3) * xix * xiy;
  q->a[6] = (1. / 3) * xiy * xiz;
  q->a[7] = (1. / 3) * xix * xiz;
  q->b[1] = (4. / 3) * etx * etx + ety * ety + etz * etz;
  q->b[2] = etx * etx + (4. / 3) * ety * ety + etz * etz;
  q->b[3] = etx * etx + ety * ety + (4. / 3) * etz * etz;
  q->b[4] = etx * etx + ety * ety + etz * etz;
  q->b[5] = (1. / 3) * etx * ety;
  q->b[6] = (1. / 3) * ety * etz;
  q->b[7] = (1. / 3) * etx * etz;
  q->c[1] = (4. / 3) * ztx * ztx + zty * zty + ztz * ztz;
  q->c[2] = ztx * ztx + (4. / 3) * zty * zty + ztz * ztz;
  q->c[3] = ztx * ztx + zty * zty + (4. / 3) * ztz * ztz;
  q->c[4] = ztx * ztx + zty * zty + ztz * ztz;
  q->c[5] = (1. / 3) * ztx * zty;
  q->c[6] = (1. / 3) * zty * ztz;
  q->c[7] = (1. / 3) * ztx * ztz;
  q->d[1] = (4. / 3) * xix * etx + xiy * ety + xiz * etz;
  q->d[2] = xix * etx + (4. / 3) * xiy * ety + xiz * etz;
  q->d[3] = xix * etx + xiy * ety + (4. / 3) * xiz * etz;
  q->d[4] = xix * etx + xiy * ety + xiz * etz;
  q->d[5] = xix * ety - (2. / 3) * xiy * etx;
  q->d[6] = xix * etz - (2. / 3) * xiz * etx;
  q->d[7] = xiy * etx - (2. / 3) * xix * ety;
  q->d[8] = xiy * etz - (2. / 3) * xiz * ety;
  q->d[9] = xiz * etx - (2. / 3) * xix * etz;
  q->d[10] = xiz * ety - (2. / 3) * xiy * etz;
  q->e[1] = (4. / 3) * xix * ztx + xiy * zty + xiz * ztz;
  q->e[2] = xix * ztx + (4. / 3) * xiy * zty + xiz * ztz;
  q->e[3] = xix * ztx + xiy * zty + (4. / 3) * xiz * ztz;
  q->e[4] = xix * ztx + xiy * zty + xiz * ztz;
  q->e[5] = xix * zty - (2. / 3) * xiy * ztx;
  q->e[6] = xix * ztz - (2. / 3) * xiz * ztx;
  q->e[7] = xiy * ztx - (2. / 3) * xix * zty;
  q->e[8] = xiy * ztz - (2. / 3) * xiz * zty;
  q->e[9] = xiz * ztx - (2. / 3) * xix * ztz;
  q->e[10] = xiz * zty - (2. / 3) * xiy * ztz;
  q->f[1] = (4. / 3) * etx * ztx + ety * zty + etz * ztz;
  q->f[2] = etx * ztx + (4. / 3) * ety * zty + etz * ztz;
  q->f[3] = etx * ztx + ety * zty + (4. / 3) * etz * ztz;
  q->f[4] = etx * ztx + ety * zty + etz * ztz;
  q->f[5] = etx * zty - (2. / 3) * ety * ztx;
  q->f[6] = etx * ztz - (2. / 3) * etz * ztx;
  q->f[7] = ety * ztx - (2. / 3) * etx * zty;
  q->f[8] = ety * ztz - (2. / 3) * etz * zty;
  q->f[9] = etz * ztx - (2. / 3) * etx * ztz;
  q->f[10] = etz * zty - (2. / 3) * ety * ztz;
}

static inline double sutherland(double mu, double T) {
  return mu * pow((T / 298.0592), 1.5) * (298.0592 + 110.) / (T + 110.);
}

/* the three faces i-1/2, j-1/2, k-1/2 of cell (i,j,k) */
static void viscous_cell(or_state *s, int i, int j, int k) {
  const size_t di = (size_t)s->Y * s->Z, dj = s->Z;
  const size_t c = IX(s, i, j, k);
  const double invXI = 1. / (s->p.dxi), invET = 1. / (s->p.det), invZT = 1. / (s->p.dzt);
  const double inv4XI = 1. / (4 * s->p.dxi), inv4ET = 1. / (4 * s->p.det), inv4ZT = 1. / (4 * s->p.dzt);
  const double Pr = s->p.pr, mu_L = s->p.mu, CvK = CV * KG;
  vprim o = vp_at(s, c);
  vprim iJ = vp_at(s, c - di + dj), iK = vp_at(s, c - di + 1), jI = vp_at(s, c + di - dj),
        kI = vp_at(s, c + di - 1), jK = vp_at(s, c - dj + 1), kJ = vp_at(s, c + dj - 1),
        im = vp_at(s, c - di), jm = vp_at(s, c - dj), km = vp_at(s, c - 1),
        ijm = vp_at(s, c - di - dj), jkm = vp_at(s, c - dj - 1), ikm = vp_at(s, c - di - 1),
        ip = vp_at(s, c + di), jp = vp_at(s, c + dj), kp = vp_at(s, c + 1);
  double U = o.U, V = o.V, W = o.W, T = o.T;
  double du_dx, dv_dx, dw_dx, du2_dx, dv2_dx, dw2_dx, duv_dx, dvw_dx, duw_dx, dT_dx;
  double du_dy, dv_dy, dw_dy, du2_dy, dv2_dy, dw2_dy, duv_dy, dvw_dy, duw_dy, dT_dy;
  double du_dz, dv_dz, dw_dz, du2_dz, dv2_dz, dw2_dz, duv_dz, dvw_dz, duw_dz, dT_dz;
  double x9[9];
  mcoef q;
  double mu_E, Ux, Vx, Wx, Tx;

  /* x-face i-1/2: Viscous_terms.cpp:399-546 */
  du_dx = (U - im.U) * invXI; dv_dx = (V - im.V) * invXI; dw_dx = (W - im.W) * invXI;
  du2_dx = (U * U - im.U * im.U) * invXI; dv2_dx = (V * V - im.V * im.V) * invXI; dw2_dx = (W * W - im.W * im.W) * invXI;
  duv_dx = (U * V - im.U * im.V) * invXI; dvw_dx = (V * W - im.V * im.W) * invXI; duw_dx = (U * W - im.U * im.W) * invXI;
  dT_dx = (T - im.T) * invXI;
  du_dy = (jp.U + iJ.U - jm.U - ijm.U) * inv4ET; dv_dy = (jp.V + iJ.V - jm.V - ijm.V) * inv4ET; dw_dy = (jp.W + iJ.W - jm.W - ijm.W) * inv4ET;
  du2_dy = (jp.U * jp.U + iJ.U * iJ.U - jm.U * jm.U - ijm.U * ijm.U) * inv4ET;
  dv2_dy = (jp.V * jp.V + iJ.V * iJ.V - jm.V * jm.V - ijm.V * ijm.V) * inv4ET;
  dw2_dy = (jp.W * jp.W + iJ.W * iJ.W - jm.W * jm.W - ijm.W * ijm.W) * inv4ET;
  duv_dy = (jp.U * jp.V + iJ.U * iJ.V - jm.U * jm.V - ijm.U * ijm.V) * inv4ET;
  dvw_dy = (jp.V * jp.W + iJ.V * iJ.W - jm.V * jm.W - ijm.V * ijm.W) * inv4ET;
  duw_dy = (jp.U * jp.W + iJ.U * iJ.W - jm.U * jm.W - ijm.U * ijm.W) * inv4ET;
  dT_dy = (jp.T + iJ.T - jm.T - ijm.T) * inv4ET;
  du_dz = (kp.U + iK.U - km.U - ikm.U) * inv4ZT; dv_dz = (kp.V + iK.V - km.V - ikm.V) * inv4ZT; dw_dz = (kp.W + iK.W - km.W - ikm.W) * inv4ZT;
  du2_dz = (kp.U * kp.U + iK.U * iK.U - km.U * km.U - ikm.U * ikm.U) * inv4ZT;
  dv2_dz = (kp.V * kp.V + iK.V * iK.V - km.V * km.V - ikm.V * ikm.V) * inv4ZT;
  dw2_dz = (kp.W * kp.W + iK.W * iK.W - km.W * km.W - ikm.W * ikm.W) * inv4ZT;
  duv_dz = (kp.U * kp.V + iK.U * iK.V - km.U * km.V - ikm.U * ikm.V) * inv4ZT;
  dvw_dz = (kp.V * kp.W + iK.V * iK.W - km.V * km.W - ikm.V * ikm.W) * inv4ZT;
  duw_dz = (kp.U * kp.W + iK.U * iK.W - km.U * km.W - ikm.U * ikm.W) * inv4ZT;
  dT_dz = (kp.T + iK.T - km.T - ikm.T) * inv4ZT;
  size_t f = IX(s, i - 1, j - 1, k - 1);
  for (int v = 0; v < 9; v++) x9[v] = s->mf[0][v][f];
  metric_products(x9, &q);
  Ux = 0.5 * (U + im.U); Vx = 0.5 * (V + im.V); Wx = 0.5 * (W + im.W); Tx = 0.5 * (T + im.T);
  mu_E = sutherland(mu_L, Tx);
  {
    double Jf = s->Jf[0][f];
    double *a = q.a, *d = q.d, *e = q.e;
    s->visc[0][0][c] = mu_E * (a[1] * du_dx + a[5] * dv_dx + a[7] * dw_dx + d[1] * du_dy + d[7] * dv_dy + d[9] * dw_dy +
                               e[1] * du_dz + e[7] * dv_dz + e[9] * dw_dz) / Jf;
    s->visc[0][1][c] = mu_E * (a[5] * du_dx + a[2] * dv_dx + a[6] * dw_dx + d[5] * du_dy + d[2] * dv_dy + d[10] * dw_dy +
                               e[5] * du_dz + e[2] * dv_dz + e[10] * dw_dz) / Jf;
    s->visc[0][2][c] = mu_E * (a[7] * du_dx + a[6] * dv_dx + a[3] * dw_dx + d[6] * du_dy + d[8] * dv_dy + d[3] * dw_dy +
                               e[6] * du_dz + e[8] * dv_dz + e[3] * dw_dz) / Jf;
    s->visc[0][3][c] = mu_E * (0.5 * a[1] * du2_dx + 0.5 * a[2] * dv2_dx + 0.5 * a[3] * dw2_dx + a[5] * duv_dx + a[6] * dvw_dx + a[7] * duw_dx + CvK * a[4] * dT_dx / (Pr) +
                               0.5 * d[1] * du2_dy + 0.5 * d[2] * dv2_dy + 0.5 * d[3] * dw2_dy + d[5] * Vx * du_dy + d[6] * Wx * du_dy + d[7] * Ux * dv_dy + d[8] * Wx * dv_dy + d[9] * Ux * dw_dy + d[10] * Vx * dw_dy + CvK * d[4] * dT_dy / (Pr) +
                               0.5 * e[1] * du2_dz + 0.5 * e[2] * dv2_dz + 0.5 * e[3] * dw2_dz + e[5] * Vx * du_dz + e[6] * Wx * du_dz + e[7] * Ux * dv_dz + e[8] * Wx * dv_dz + e[9] * Ux * dw_dz + e[10] * Vx * dw_dz + CvK * e[4] * dT_dz / (Pr)) / Jf;
  }

  /* y-face j-1/2: Viscous_terms.cpp:549-700 */
  du_dx = (ip.U + jI.U - im.U - ijm.U) * inv4XI; dv_dx = (ip.V + jI.V - im.V - ijm.V) * inv4XI; dw_dx = (ip.W + jI.W - im.W - ijm.W) * inv4XI;
  du2_dx = (ip.U * ip.U + jI.U * jI.U - im.U * im.U - ijm.U * ijm.U) * inv4XI;
  dv2_dx = (ip.V * ip.V + jI.V * jI.V - im.V * im.V - ijm.V * ijm.V) * inv4XI;
  dw2_dx = (ip.W * ip.W + jI.W * jI.W - im.W * im.W - ijm.W * ijm.W) * inv4XI;
  duv_dx = (ip.U * ip.V + jI.U * jI.V - im.U * im.V - ijm.U * ijm.V) * inv4XI;
  dvw_dx = (ip.V * ip.W + jI.V * jI.W - im.V * im.W - ijm.V * ijm.W) * inv4XI;
  duw_dx = (ip.U * ip.W + jI.U * jI.W - im.U * im.W - ijm.U * ijm.W) * inv4XI;
  dT_dx = (ip.T + jI.T - im.T - ijm.T) * inv4XI;
  du_dy = (U - jm.U) * invET; dv_dy = (V - jm.V) * invET; dw_dy = (W - jm.W) * invET;
  du2_dy = (U * U - jm.U * jm.U) * invET; dv2_dy = (V * V - jm.V * jm.V) * invET; dw2_dy = (W * W - jm.W * jm.W) * invET;
  duv_dy = (U * V - jm.U * jm.V) * invET; dvw_dy = (V * W - jm.V * jm.W) * invET; duw_dy = (U * W - jm.U * jm.W) * invET;
  dT_dy = (T - jm.T) * invET;
  du_dz = (kp.U + jK.U - km.U - jkm.U) * inv4ZT; dv_dz = (kp.V + jK.V - km.V - jkm.V) * inv4ZT; dw_dz = (kp.W + jK.W - km.W - jkm.W) * inv4ZT;
  du2_dz = (kp.U * kp.U + jK.U * jK.U - km.U * km.U - jkm.U * jkm.U) * inv4ZT;
  dv2_dz = (kp.V * kp.V + jK.V * jK.V - km.V * km.V - jkm.V * jkm.V) * inv4ZT;
  dw2_dz = (kp.W * kp.W + jK.W * jK.W - km.W * km.W - jkm.W * jkm.W) * inv4ZT;
  duv_dz = (kp.U * kp.V + jK.U * jK.V - km.U * km.V - jkm.U * jkm.V) * inv4ZT;
  dvw_dz = (kp.V * kp.W + jK.V * jK.W - km.V * km.W - jkm.V * jkm.W) * inv4ZT;
  duw_dz = (kp.U * kp.W + jK.U * jK.W - km.U * km.W - jkm.U * jkm.W) * inv4ZT;
  dT_dz = (kp.T + jK.T - km.T - jkm.T) * inv4ZT;
  for (int v = 0; v < 9; v++) x9[v] = s->mf[1][v][f];
  metric_products(x9, &q);
  double Uy = 0.5 * (U + jm.U), Vy = 0.5 * (V + jm.V), Wy = 0.5 * (W + jm.W), Ty = 0.5 * (T + jm.T);
  mu_E = sutherland(mu_L, Ty);
  {
    double Jf = s->Jf[1][f];
    double *b = q.b, *d = q.d, *fm = q.f;
    s->visc[1][0][c] = mu_E * (d[1] * du_dx + d[5] * dv_dx + d[6] * dw_dx + b[1] * du_dy + b[5] * dv_dy + b[7] * dw_dy +
                               fm[1] * du_dz + fm[7] * dv_dz + fm[9] * dw_dz) / Jf;
    s->visc[1][1][c] = mu_E * (d[7] * du_dx + d[2] * dv_dx + d[8] * dw_dx + b[5] * du_dy + b[2] * dv_dy + b[6] * dw_dy +
                               fm[5] * du_dz + fm[2] * dv_dz + fm[10] * dw_dz) / Jf;
    s->visc[1][2][c] = mu_E * (d[9] * du_dx + d[10] * dv_dx + d[3] * dw_dx + b[7] * du_dy + b[6] * dv_dy + b[3] * dw_dy +
                               fm[6] * du_dz + fm[8] * dv_dz + fm[3] * dw_dz) / Jf;
    s->visc[1][3][c] = mu_E * (0.5 * b[1] * du2_dy + 0.5 * b[2] * dv2_dy + 0.5 * b[3] * dw2_dy + b[5] * duv_dy + b[6] * dvw_dy + b[7] * duw_dy + CvK * b[4] * dT_dy / (Pr) +
                               0.5 * d[1] * du2_dx + 0.5 * d[2] * dv2_dx + 0.5 * d[3] * dw2_dx + d[5] * Uy * dv_dx + d[6] * Uy * dw_dx + d[7] * Vy * du_dx + d[8] * Vy * dw_dx + d[9] * Wy * du_dx + d[10] * Wy * dv_dx + CvK * d[4] * dT_dx / (Pr) +
                               0.5 * fm[1] * du2_dz + 0.5 * fm[2] * dv2_dz + 0.5 * fm[3] * dw2_dz + fm[5] * Vy * du_dz + fm[6] * Wy * du_dz + fm[7] * Uy * dv_dz + fm[8] * Wy * dv_dz + fm[9] * Uy * dw_dz + fm[10] * Vy * dw_dz + CvK * fm[4] * dT_dz / (Pr)) / Jf;
  }

  /* z-face k-1/2: Viscous_terms.cpp:714-861, including the typo of :744-746
   * that pairs u at (i,j+1,k-1) with v, w at (i-1,j+1,k) */
  du_dx = (ip.U + kI.U - im.U - ikm.U) * inv4XI; dv_dx = (ip.V + kI.V - im.V - ikm.V) * inv4XI; dw_dx = (ip.W + kI.W - im.W - ikm.W) * inv4XI;
  du2_dx = (ip.U * ip.U + kI.U * kI.U - im.U * im.U - ikm.U * ikm.U) * inv4XI;
  dv2_dx = (ip.V * ip.V + kI.V * kI.V - im.V * im.V - ikm.V * ikm.V) * inv4XI;
  dw2_dx = (ip.W * ip.W + kI.W * kI.W - im.W * im.W - ikm.W * ikm.W) * inv4XI;
  duv_dx = (ip.U * ip.V + kI.U * kI.V - im.U * im.V - ikm.U * ikm.V) * inv4XI;
  dvw_dx = (ip.V * ip.W + kI.V * kI.W - im.V * im.W - ikm.V * ikm.W) * inv4XI;
  duw_dx = (ip.U * ip.W + kI.U * kI.W - im.U * im.W - ikm.U * ikm.W) * inv4XI;
  dT_dx = (ip.T + kI.T - im.T - ikm.T) * inv4XI;
  du_dy = (jp.U + kJ.U - jm.U - jkm.U) * inv4ET; dv_dy = (jp.V + kJ.V - jm.V - jkm.V) * inv4ET; dw_dy = (jp.W + kJ.W - jm.W - jkm.W) * inv4ET;
  du2_dy = (jp.U * jp.U + kJ.U * kJ.U - jm.U * jm.U - jkm.U * jkm.U) * inv4ET;
  dv2_dy = (jp.V * jp.V + kJ.V * kJ.V - jm.V * jm.V - jkm.V * jkm.V) * inv4ET;
  dw2_dy = (jp.W * jp.W + kJ.W * kJ.W - jm.W * jm.W - jkm.W * jkm.W) * inv4ET;
  duv_dy = (jp.U * jp.V + kJ.U * iJ.V - jm.U * jm.V - jkm.U * jkm.V) * inv4ET;
  dvw_dy = (jp.V * jp.W + kJ.V * iJ.W - jm.V * jm.W - jkm.V * jkm.W) * inv4ET;
  duw_dy = (jp.U * jp.W + kJ.U * iJ.W - jm.U * jm.W - jkm.U * jkm.W) * inv4ET;
  dT_dy = (jp.T + kJ.T - jm.T - jkm.T) * inv4ET;
  du_dz = (U - km.U) * invZT; dv_dz = (V - km.V) * invZT; dw_dz = (W - km.W) * invZT;
  du2_dz = (U * U - km.U * km.U) * invZT; dv2_dz = (V * V - km.V * km.V) * invZT; dw2_dz = (W * W - km.W * km.W) * invZT;
  duv_dz = (U * V - km.U * km.V) * invZT; dvw_dz = (V * W - km.V * km.W) * invZT; duw_dz = (U * W - km.U * km.W) * invZT;
  dT_dz = (T - km.T) * invZT;
  for (int v = 0; v < 9; v++) x9[v] = s->mf[2][v][f];
  metric_products(x9, &q);
  double Uz = 0.5 * (U + km.U), Vz = 0.5 * (V + km.V), Wz = 0.5 * (W + km.W), Tz = 0.5 * (T + km.T);
  mu_E = sutherland(mu_L, Tz);
  {
    double Jf = s->Jf[2][f];
    double *c_ = q.c, *e = q.e, *fm = q.f;
    s->visc[2][0][c] = mu_E * (e[1] * du_dx + e[5] * dv_dx + e[6] * dw_dx + fm[1] * du_dy + fm[5] * dv_dy + fm[6] * dw_dy +
                               c_[1] * du_dz + c_[5] * dv_dz + c_[7] * dw_dz) / Jf;
    s->visc[2][1][c] = mu_E * (e[7] * du_dx + e[2] * dv_dx + e[8] * dw_dx + fm[7] * du_dy + fm[2] * dv_dy + fm[8] * dw_dy +
                               c_[5] * du_dz + c_[2] * dv_dz + c_[6] * dw_dz) / Jf;
    s->visc[2][2][c] = mu_E * (e[9] * du_dx + e[10] * dv_dx + e[3] * dw_dx + fm[9] * du_dy + fm[10] * dv_dy + fm[3] * dw_dy +
                               c_[7] * du_dz + c_[6] * dv_dz + c_[3] * dw_dz) / Jf;
    s->visc[2][3][c] = mu_E * (0.5 * c_[1] * du2_dz + 0.5 * c_[2] * dv2_dz + 0.5 * c_[3] * dw2_dz + c_[5] * duv_dz + c_[6] * dvw_dz + c_[7] * duw_dz + CvK * c_[4] * dT_dz / (Pr) +
                               0.5 * e[1] * du2_dx + 0.5 * e[2] * dv2_dx + 0.5 * e[3] * dw2_dx + e[5] * Uz * dv_dx + e[6] * Uz * dw_dx + e[7] * Vz * du_dx + e[8] * Vz * dw_dx + e[9] * Wz * du_dx + e[10] * Wz * dv_dx + CvK * e[4] * dT_dx / (Pr) +
                               0.5 * fm[1] * du2_dy + 0.5 * fm[2] * dv2_dy + 0.5 * fm[3] * dw2_dy + fm[5] * Uz * dv_dy + fm[6] * Uz * dw_dy + fm[7] * Vz * du_dy + fm[8] * Vz * dw_dy + fm[9] * Wz * du_dy + fm[10] * Wz * dv_dy + CvK * fm[4] * dT_dy / (Pr)) / Jf;
  }
}

void or_viscous(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1, nyy = jn + 1, nzz = kn + 1;
  const size_t di = (size_t)s->Y * s->Z, dj = s->Z;
  const double invXI = 1. / (s->p.dxi), invET = 1. / (s->p.det), invZT = 1. / (s->p.dzt);
  for (int i = 3; i <= ie + 1; i++)
    for (int j = 2; j <= nyy; j++)
      for (int k = 2; k <= nzz; k++) viscous_cell(s, i, j, k);
  /* divergence, Viscous_terms.cpp:875-904 */
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        for (int v = 0; v < 4; v++)
          s->vF[v][c] = (s->visc[0][v][c + di] - s->visc[0][v][c]) * invXI +
                        (s->visc[1][v][c + dj] - s->visc[1][v][c]) * invET +
                        (s->visc[2][v][c + 1] - s->visc[2][v][c]) * invZT;
      }
}

/* ------------------------------------------------------------------------ */
/* dual-time residual, LU-SGS sweeps, update: Dual_time_stepping.cpp         */

typedef struct { double rho, u, v, w, VV, P, C, T, H, beta; } cprim;

static inline cprim cp_at(const or_state *s, size_t c) {
  cprim r;
  const double J = s->J[c];
  r.rho = s->U_[0][c] * J;
  r.u = s->U_[1][c] / s->U_[0][c];
  r.v = s->U_[2][c] / s->U_[0][c];
  r.w = s->U_[3][c] / s->U_[0][c];
  r.VV = r.u * r.u + r.v * r.v + r.w * r.w;
  r.P = (s->U_[4][c] * J - 0.5 * r.rho * r.VV) * (KG - 1);
  r.C = KG * r.P / r.rho;
  r.T = r.P / r.rho;
  r.H = 0.5 * r.VV + r.C / (KG - 1);
  r.beta = MAX(r.VV / r.C, s->p.e);
  return r;
}

/* the cell's own LU-SGS diagonal, Dual_time_stepping.cpp:853-895 */
typedef struct { double d11, d22, d51; } diag3;

static inline diag3 diag_at(const or_state *s, size_t c, const cprim *q) {
  double xix = s->m[0][c], xiy = s->m[1][c], xiz = s->m[2][c];
  double etx = s->m[3][c], ety = s->m[4][c], etz = s->m[5][c];
  double ztx = s->m[6][c], zty = s->m[7][c], ztz = s->m[8][c];
  double beta = q->beta, C = q->C, deltaT = s->p.dt;
  double U = xix * q->u + xiy * q->v + xiz * q->w;
  double V = etx * q->u + ety * q->v + etz * q->w;
  double W = ztx * q->u + zty * q->v + ztz * q->w;
  double Sx = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * C * (xix * xix + xiy * xiy + xiz * xiz));
  double Sy = sqrt(V * V * (beta - 1) * (beta - 1) + 4 * beta * C * (etx * etx + ety * ety + etz * etz));
  double Sz = sqrt(W * W * (beta - 1) * (beta - 1) + 4 * beta * C * (ztx * ztx + zty * zty + ztz * ztz));
  double lambdaX = ((beta + 1) * fabs(U) + Sx) / 2;
  double lambdaY = ((beta + 1) * fabs(V) + Sy) / 2;
  double lambdaZ = ((beta + 1) * fabs(W) + Sz) / 2;
  double lambda = lambdaX / s->p.dxi + lambdaY / s->p.det + lambdaZ / s->p.dzt;
  diag3 d;
  d.d11 = 2 * deltaT / (3 * beta + 2 * lambda * deltaT);
  d.d22 = 2 * deltaT / (3 + 2 * lambda * deltaT);
  double temp1 = 6 * (KG - 1) * (beta - 1) * deltaT;
  double temp2 = KG * (3 + 2 * lambda * deltaT) * (3 * beta + 2 * lambda * deltaT) * q->rho;
  d.d51 = -temp1 / temp2;
  return d;
}

/* split Jacobian of one neighbour in one direction, Dual_time_stepping.cpp:
 * 1021-1170 (A+, B+, C+) and :1404-1524 (A-, B-, C- diagonals).  `xorder`
 * selects the x-direction product order of row 5 (Aplus52 = 0.5*xix*beta*
 * T*(K-1)) against the y/z order (Bplus52 = 0.5*beta*T*(K-1)*etx). */
typedef struct { double p11, p12, p13, p14, p21, p22, p31, p41, p51, p52, p53, p54, m11, m22; } splitj;

static inline splitj split_at(const or_state *s, size_t c, int dir) {
  cprim q = cp_at(s, c);
  double mx = s->m[3 * dir][c], my = s->m[3 * dir + 1][c], mz = s->m[3 * dir + 2][c];
  double beta = q.beta, U = mx * q.u + my * q.v + mz * q.w;
  double Sx = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * q.C * (mx * mx + my * my + mz * mz));
  double lambdaX = ((beta + 1) * fabs(U) + Sx) / 2;
  double d = fabs(lambdaX);
  splitj a;
  a.p11 = 0.5 * (beta * U + d);
  a.p12 = 0.5 * q.P * KG * beta * mx;
  a.p13 = 0.5 * q.P * KG * beta * my;
  a.p14 = 0.5 * q.P * KG * beta * mz;
  a.p21 = 0.5 * mx / q.rho;
  a.p22 = 0.5 * (U + d);
  a.p31 = 0.5 * my / q.rho;
  a.p41 = 0.5 * mz / q.rho;
  a.p51 = 0.5 * U * (KG - 1) * (beta - 1) / q.rho / KG;
  if (dir == 0) {
    a.p52 = 0.5 * mx * beta * q.T * (KG - 1);
    a.p53 = 0.5 * my * beta * q.T * (KG - 1);
    a.p54 = 0.5 * mz * beta * q.T * (KG - 1);
  } else {
    a.p52 = 0.5 * beta * q.T * (KG - 1) * mx;
    a.p53 = 0.5 * beta * q.T * (KG - 1) * my;
    a.p54 = 0.5 * beta * q.T * (KG - 1) * mz;
  }
  a.m11 = 0.5 * (beta * U - d);
  a.m22 = 0.5 * (U - d);
  return a;
}

/* sponge layers, Dual_time_stepping.cpp:327-664: the Residual arrays are
 * zeroed, then the first nx_inlet and the last nx_outlet interior planes of
 * the x extent (an open slab is the whole extent) get the absorbing terms.
 * The inlet profile uses the slab's first global index where the outlet one
 * uses the plane's (:586 against :644).  The outlet target velocity is the
 * volume mean of u over plane 3, rows 2..Ny+2 and 2..Nz+2 (:510-532). */
static void or_sponge(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1, nyy = jn + 1, nzz = kn + 1;
  const size_t n = or_n(s);
  for (int v = 0; v < 5; v++) memset(s->spg[v], 0, n * sizeof(double));
  if (!s->p.x_open) return;
  const int nxin = s->p.nx_inlet, nxout = s->p.nx_outlet, Xout = s->p.nx, gstart = 0;
  const double dXI = s->p.dxi, dET = s->p.det, dZT = s->p.dzt, high = s->high, e = s->p.e;
  double z1 = 0.0;
  const double DZ = 1. / (high * dZT * s->p.nz);
  for (int j = 2; j <= nyy; j++)
    for (int k = 2; k <= nzz; k++) {
      size_t c = IX(s, 3, j, k);
      double U = s->U_[1][c] / s->U_[0][c];
      z1 = z1 + U * dET / s->m[4][c] * dZT;
    }
  const double targetU = z1 * DZ;
  const double U_in_0 = 1.0, Sigma_in_0 = 0.035, U_out_0 = 1.0, Sigma_out_0 = 1.25;
  for (int side = 0; side < 2; side++) {
    int i0, i1;
    if (!side) {
      if (!(gstart < nxin)) continue;
      i0 = 3; i1 = (Xout - 1 < nxin) ? ie : nxin - gstart + 2;
    } else {
      if (!(Xout - 1 > Xout - nxout - 1)) continue;
      i0 = (gstart > Xout - nxout - 1) ? 3 : (Xout - nxout) - gstart + 2;
      i1 = ie;
    }
    for (int i = i0; i <= i1; i++)
      for (int j = 2; j <= jn; j++)
        for (int k = 2; k <= kn; k++) {
          size_t c = IX(s, i, j, k), b = c - (size_t)s->Y * s->Z;
          double **q = s->U_;
          const double *J = s->J;
          double rho = q[0][c] * J[c];
          double u = q[1][c] / q[0][c];
          double v = q[2][c] / q[0][c];
          double w = q[3][c] / q[0][c];
          double VV = u * u + v * v + w * w;
          double P = (q[4][c] * J[c] - 0.5 * rho * VV) * (KG - 1);
          double C = KG * P / rho;
          double beta = MAX(VV / C, e);
          double C_plan = 0.5 * sqrt(u * u * (beta - 1) * (beta - 1) + 4 * beta * C);
          double Us, Sig, t2 = 0, t5 = 0;
          if (!side) {
            Us = pow((((nxin - gstart - 0.5) * 1.0) / nxin), 3.0) * U_in_0 * C_plan;
            Sig = Sigma_in_0 * Us / high;
          } else {
            /* nx of Resolution.h is X_out + 1 */
            Us = pow((((i + gstart - 0.5 - ((Xout + 1) - nxout)) * 1.0) / nxout), 3.0) * U_out_0 * C_plan;
            Sig = Sigma_out_0 * Us / high;
            t2 = 1.1842 * targetU;
            t5 = 0.5 * 1.1842 * targetU * targetU;
          }
          double **sp = s->spg;
          sp[0][c] = -Us * (q[0][c] * J[c] - q[0][b] * J[b]) / dXI - Sig * (rho - 1.1842);
          sp[1][c] = -Us * (q[1][c] * J[c] - q[1][b] * J[b]) / dXI - Sig * (side ? rho * u - t2 : rho * u);
          sp[2][c] = -Us * (q[2][c] * J[c] - q[2][b] * J[b]) / dXI - Sig * (rho * v);
          sp[3][c] = -Us * (q[3][c] * J[c] - q[3][b] * J[b]) / dXI - Sig * (rho * w);
          sp[4][c] = -Us * (q[4][c] * J[c] - q[4][b] * J[b]) / dXI -
                     Sig * (side ? q[4][c] * J[c] - 253250.0 - t5 : q[4][c] * J[c] - 253250.0);
        }
  }
}

/* residual assembly, Dual_time_stepping.cpp:737-922; with dplusgs, that of
 * DPLUSGS.cpp:324-478, which has no sponge terms and always the uniform
 * force */
static void dts_residual(or_state *s, int dplusgs) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1, nyy = jn + 1, nzz = kn + 1;
  const double deltaT = s->p.dt, dXI = s->p.dxi, dET = s->p.det, dZT = s->p.dzt;
  /* ghost rows of NL/NR are zero, :255-323 */
  for (int i = 2; i <= ie + 1; i++) {
    for (int k = 1; k <= nzz; k++)
      for (int v = 0; v < 5; v++) {
        s->NL[v][IX(s, i, 1, k)] = 0; s->NR[v][IX(s, i, 1, k)] = 0;
        s->NL[v][IX(s, i, nyy, k)] = 0; s->NR[v][IX(s, i, nyy, k)] = 0;
      }
    for (int j = 1; j <= nyy; j++)
      for (int v = 0; v < 5; v++) {
        s->NL[v][IX(s, i, j, 1)] = 0; s->NR[v][IX(s, i, j, 1)] = 0;
        s->NL[v][IX(s, i, j, nzz)] = 0; s->NR[v][IX(s, i, j, nzz)] = 0;
      }
  }
  if (s->p.x_open)   /* :204-246: the end planes of the first and last rank */
    for (int side = 0; side < 2; side++) {
      int ig = side ? ie + 1 : 2;
      for (int j = 1; j <= nyy; j++)
        for (int k = 1; k <= nzz; k++)
          for (int v = 0; v < 5; v++) { s->NL[v][IX(s, ig, j, k)] = 0; s->NR[v][IX(s, ig, j, k)] = 0; }
    }
  or_sponge(s);
  if (dplusgs)
    for (int v = 0; v < 5; v++) memset(s->spg[v], 0, or_n(s) * sizeof(double));
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j < nyy; j++)
      for (int k = 2; k < nzz; k++) {
        size_t c = IX(s, i, j, k);
        const double J = s->J[c];
        cprim q = cp_at(s, c);
        double rho = q.rho, u = q.u, v = q.v, w = q.w, VV = q.VV, T = q.T, H = q.H, beta = q.beta;
        double temp = rho * KG;
        double d11 = -(H * (KG - 1) + VV - KG * (T + VV)) * beta;
        double d12 = -(KG - 1) * u * beta, d13 = -(KG - 1) * v * beta, d14 = -(KG - 1) * w * beta;
        double d15 = (KG - 1) * beta;
        double d21 = -u / rho, d22 = 1 / rho, d23 = 0, d24 = 0, d25 = 0;
        double d31 = -v / rho, d32 = 0, d33 = 1 / rho, d34 = 0, d35 = 0;
        double d41 = -w / rho, d42 = 0, d43 = 0, d44 = 1 / rho, d45 = 0;
        double d51 = (KG - 1) * (VV + KG * T * beta + (KG - 1) * VV * beta + H * (-1 + beta - KG * beta)) / temp;
        double d52 = -(KG - 1) * u * (1 + (KG - 1) * beta) / temp;
        double d53 = -(KG - 1) * v * (1 + (KG - 1) * beta) / temp;
        double d54 = -(KG - 1) * w * (1 + (KG - 1) * beta) / temp;
        double d55 = (KG - 1) * (1 + (KG - 1) * beta) / temp;
        double Rp[5], Rf[5], Rk[5];
        size_t fx1 = IX(s, i, j - 1, k - 1), fx0 = IX(s, i - 1, j - 1, k - 1);
        size_t fy1 = IX(s, i - 1, j, k - 1), fy0 = IX(s, i - 1, j - 1, k - 1);
        size_t fz1 = IX(s, i - 1, j - 1, k), fz0 = IX(s, i - 1, j - 1, k - 1);
        for (int n = 0; n < 5; n++) {
          Rp[n] = -(3 * s->U_[n][c] - 4 * s->U[n][c] + s->Uq[n][c]) / (2 * deltaT);
          Rf[n] = -((s->inF[0][n][fx1] - s->inF[0][n][fx0]) / dXI +
                    (s->inF[1][n][fy1] - s->inF[1][n][fy0]) / dET +
                    (s->inF[2][n][fz1] - s->inF[2][n][fz0]) / dZT);
        }
        double f = (s->p.buoyancy && !dplusgs) ? -(rho - 1.1842) * 9.81 : s->p.force;   /* :831 */
        double **sp = s->spg;
        Rk[0] = sp[0][c] / J + Rp[0] + Rf[0];
        Rk[1] = sp[1][c] / J + Rp[1] + Rf[1] + s->vF[0][c] + f / J;
        Rk[2] = sp[2][c] / J + Rp[2] + Rf[2] + s->vF[1][c];
        Rk[3] = sp[3][c] / J + Rp[3] + Rf[3] + s->vF[2][c];
        Rk[4] = sp[4][c] / J + Rp[4] + Rf[4] + s->vF[3][c] + f * u / J;
        double MR1 = (d11 * Rk[0] + d12 * Rk[1] + d13 * Rk[2] + d14 * Rk[3] + d15 * Rk[4]);
        double MR2 = (d21 * Rk[0] + d22 * Rk[1] + d23 * Rk[2] + d24 * Rk[3] + d25 * Rk[4]);
        double MR3 = (d31 * Rk[0] + d32 * Rk[1] + d33 * Rk[2] + d34 * Rk[3] + d35 * Rk[4]);
        double MR4 = (d41 * Rk[0] + d42 * Rk[1] + d43 * Rk[2] + d44 * Rk[3] + d45 * Rk[4]);
        double MR5 = (d51 * Rk[0] + d52 * Rk[1] + d53 * Rk[2] + d54 * Rk[3] + d55 * Rk[4]);
        s->MR[0][c] = MR1; s->MR[1][c] = MR2; s->MR[2][c] = MR3; s->MR[3][c] = MR4; s->MR[4][c] = MR5;
        diag3 dd = diag_at(s, c, &q);
        double n1 = dd.d11 * MR1, n2 = dd.d22 * MR2, n3 = dd.d22 * MR3, n4 = dd.d22 * MR4;
        double n5 = dd.d51 * MR1 + dd.d22 * MR5;
        s->NL[0][c] = n1; s->NL[1][c] = n2; s->NL[2][c] = n3; s->NL[3][c] = n4; s->NL[4][c] = n5;
        s->NR[0][c] = n1; s->NR[1][c] = n2; s->NR[2][c] = n3; s->NR[3][c] = n4; s->NR[4][c] = n5;
        (void)d12;
      }
  (void)dXI; (void)dET; (void)dZT;
}

void or_dts_residual(or_state *s) { dts_residual(s, 0); }
void or_dplur_residual(or_state *s) { dts_residual(s, 1); }

/* forward sweep at one cell, Dual_time_stepping.cpp:1017-1293 */
static void forward_cell(or_state *s, int i, int j, int k) {
  const size_t di = (size_t)s->Y * s->Z, dj = s->Z;
  size_t c = IX(s, i, j, k), ci = c - di, cj = c - dj, ck = c - 1;
  splitj A = split_at(s, ci, 0), B = split_at(s, cj, 1), C = split_at(s, ck, 2);
  double **NL = s->NL;
  const double dXI = s->p.dxi, dET = s->p.det, dZT = s->p.dzt;
  double LL1 = (-A.p11 * NL[0][ci] - A.p12 * NL[1][ci] - A.p13 * NL[2][ci] - A.p14 * NL[3][ci]) / dXI +
               (-B.p11 * NL[0][cj] - B.p12 * NL[1][cj] - B.p13 * NL[2][cj] - B.p14 * NL[3][cj]) / dET +
               (-C.p11 * NL[0][ck] - C.p12 * NL[1][ck] - C.p13 * NL[2][ck] - C.p14 * NL[3][ck]) / dZT;
  double LL2 = (-A.p21 * NL[0][ci] - A.p22 * NL[1][ci]) / dXI + (-B.p21 * NL[0][cj] - B.p22 * NL[1][cj]) / dET +
               (-C.p21 * NL[0][ck] - C.p22 * NL[1][ck]) / dZT;
  double LL3 = (-A.p31 * NL[0][ci] - A.p22 * NL[2][ci]) / dXI + (-B.p31 * NL[0][cj] - B.p22 * NL[2][cj]) / dET +
               (-C.p31 * NL[0][ck] - C.p22 * NL[2][ck]) / dZT;
  double LL4 = (-A.p41 * NL[0][ci] - A.p22 * NL[3][ci]) / dXI + (-B.p41 * NL[0][cj] - B.p22 * NL[3][cj]) / dET +
               (-C.p41 * NL[0][ck] - C.p22 * NL[3][ck]) / dZT;
  double LL5 = (-A.p51 * NL[0][ci] - A.p52 * NL[1][ci] - A.p53 * NL[2][ci] - A.p54 * NL[3][ci] - A.p22 * NL[4][ci]) / dXI +
               (-B.p51 * NL[0][cj] - B.p52 * NL[1][cj] - B.p53 * NL[2][cj] - B.p54 * NL[3][cj] - B.p22 * NL[4][cj]) / dET +
               (-C.p51 * NL[0][ck] - C.p52 * NL[1][ck] - C.p53 * NL[2][ck] - C.p54 * NL[3][ck] - C.p22 * NL[4][ck]) / dZT;
  cprim q = cp_at(s, c);
  diag3 d = diag_at(s, c, &q);
  NL[0][c] = d.d11 * (s->MR[0][c] - LL1);
  NL[1][c] = d.d22 * (s->MR[1][c] - LL2);
  NL[2][c] = d.d22 * (s->MR[2][c] - LL3);
  NL[3][c] = d.d22 * (s->MR[3][c] - LL4);
  NL[4][c] = d.d51 * (s->MR[0][c] - LL1) + d.d22 * (s->MR[4][c] - LL5);
}

/* backward sweep at one cell, Dual_time_stepping.cpp:1350-1655 */
static void backward_cell(or_state *s, int i, int j, int k) {
  const size_t di = (size_t)s->Y * s->Z, dj = s->Z;
  size_t c = IX(s, i, j, k), ci = c + di, cj = c + dj, ck = c + 1;
  splitj A = split_at(s, ci, 0), B = split_at(s, cj, 1), C = split_at(s, ck, 2);
  double **NR = s->NR, **NL = s->NL;
  const double dXI = s->p.dxi, dET = s->p.det, dZT = s->p.dzt;
  double UU1 = (+A.m11 * NR[0][ci] + A.p12 * NR[1][ci] + A.p13 * NR[2][ci] + A.p14 * NR[3][ci]) / dXI +
               (+B.m11 * NR[0][cj] + B.p12 * NR[1][cj] + B.p13 * NR[2][cj] + B.p14 * NR[3][cj]) / dET +
               (+C.m11 * NR[0][ck] + C.p12 * NR[1][ck] + C.p13 * NR[2][ck] + C.p14 * NR[3][ck]) / dZT;
  double UU2 = (+A.p21 * NR[0][ci] + A.m22 * NR[1][ci]) / dXI + (+B.p21 * NR[0][cj] + B.m22 * NR[1][cj]) / dET +
               (+C.p21 * NR[0][ck] + C.m22 * NR[1][ck]) / dZT;
  double UU3 = (+A.p31 * NR[0][ci] + A.m22 * NR[2][ci]) / dXI + (+B.p31 * NR[0][cj] + B.m22 * NR[2][cj]) / dET +
               (+C.p31 * NR[0][ck] + C.m22 * NR[2][ck]) / dZT;
  double UU4 = (+A.p41 * NR[0][ci] + A.m22 * NR[3][ci]) / dXI + (+B.p41 * NR[0][cj] + B.m22 * NR[3][cj]) / dET +
               (+C.p41 * NR[0][ck] + C.m22 * NR[3][ck]) / dZT;
  double UU5 = (+A.p51 * NR[0][ci] + A.p52 * NR[1][ci] + A.p53 * NR[2][ci] + A.p54 * NR[3][ci] + A.m22 * NR[4][ci]) / dXI +
               (+B.p51 * NR[0][cj] + B.p52 * NR[1][cj] + B.p53 * NR[2][cj] + B.p54 * NR[3][cj] + B.m22 * NR[4][cj]) / dET +
               (+C.p51 * NR[0][ck] + C.p52 * NR[1][ck] + C.p53 * NR[2][ck] + C.p54 * NR[3][ck] + C.m22 * NR[4][ck]) / dZT;
  cprim q = cp_at(s, c);
  diag3 d = diag_at(s, c, &q);
  NR[0][c] = NL[0][c] - d.d11 * UU1;
  NR[1][c] = NL[1][c] - d.d22 * UU2;
  NR[2][c] = NL[2][c] - d.d22 * UU3;
  NR[3][c] = NL[3][c] - d.d22 * UU4;
  NR[4][c] = NL[4][c] - (d.d51 * UU1 + d.d22 * UU5);
}

/* two symmetric sweeps with the lagged periodic x halos of NL / NR,
 * Dual_time_stepping.cpp:931-1689.  Any order that visits a cell after its
 * three upwind neighbours gives the same numbers as the reference's i+j+k
 * hyperplanes; lexicographic order is one such order. */
void or_sweeps(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  const size_t plane = (size_t)s->Y * s->Z;
  for (int sweep = 1; sweep <= 2; sweep++) {
    for (int v = 0; v < 5 && !s->p.x_open; v++) {   /* open: the end planes stay zero */
      memmove(s->NL[v] + 2 * plane, s->NL[v] + (size_t)ie * plane, plane * sizeof(double));
      memmove(s->NR[v] + (size_t)(ie + 1) * plane, s->NR[v] + 3 * plane, plane * sizeof(double));
    }
    for (int i = 3; i <= ie; i++)
      for (int j = 2; j <= jn; j++)
        for (int k = 2; k <= kn; k++) forward_cell(s, i, j, k);
    for (int i = ie; i >= 3; i--)
      for (int j = jn; j >= 2; j--)
        for (int k = kn; k >= 2; k--) backward_cell(s, i, j, k);
    for (int i = 3; i <= ie; i++)
      for (int j = 2; j <= jn; j++)
        for (int k = 2; k <= kn; k++) {
          size_t c = IX(s, i, j, k);
          for (int v = 0; v < 5; v++) s->NL[v][c] = s->NR[v][c];
        }
  }
}

/* primitive-variable update and residual norms, Dual_time_stepping.cpp:
 * 1702-1782.  er[v] = sqrt(sum of squared increments) / (Nx Ny Nz) for
 * rho, u, v, w, p/rho. */
void or_update(or_state *s, double *er) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  double e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        const double J = s->J[c];
        double **q = s->U_, **NR = s->NR;
        double rhoold = q[0][c] * J;
        double Uold = q[1][c] / q[0][c];
        double Vold = q[2][c] / q[0][c];
        double Wold = q[3][c] / q[0][c];
        double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
        double Pold = (q[4][c] * J - 0.5 * rhoold * VVold) * (KG - 1);
        double Told = Pold / rhoold;
        double P = Pold + NR[0][c] * J;
        double U = Uold + NR[1][c] * J;
        double V = Vold + NR[2][c] * J;
        double W = Wold + NR[3][c] * J;
        double T = Told + NR[4][c] * J;
        double rho = P / T;
        q[0][c] = rho / J;
        q[1][c] = rho * U / J;
        q[2][c] = rho * V / J;
        q[3][c] = rho * W / J;
        q[4][c] = (P / (KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / J;
        s->res[0][c] = (rho - rhoold) * (rho - rhoold);
        s->res[1][c] = (U - Uold) * (U - Uold);
        s->res[2][c] = (V - Vold) * (V - Vold);
        s->res[3][c] = (W - Wold) * (W - Wold);
        s->res[4][c] = (T - Told) * (T - Told);
        e1 = e1 + s->res[0][c]; e2 = e2 + s->res[1][c]; e3 = e3 + s->res[2][c];
        e4 = e4 + s->res[3][c]; e5 = e5 + s->res[4][c];
      }
  double DN = 1. / ((double)s->p.nx * s->p.ny * s->p.nz);
  er[0] = sqrt(e1) * DN; er[1] = sqrt(e2) * DN; er[2] = sqrt(e3) * DN;
  er[3] = sqrt(e4) * DN; er[4] = sqrt(e5) * DN;
}

/* ------------------------------------------------------------------------ */
/* DP-LUR inner solver: DPLUSGS.cpp (the alternative to the LU-SGS sweeps    */
/* of Dual_time_stepping, left commented out at main.cpp:268-284)             */

/* one Jacobi relaxation at one cell, DPLUSGS.cpp:560-1118: the lower and
 * upper neighbours' split Jacobians applied to the previous iterate NL, the
 * inviscid diagonal of the cell (:1068-1107), NR = D^-1 (MR - LL - UU) */
static void dplur_cell(or_state *s, int i, int j, int k) {
  const size_t di = (size_t)s->Y * s->Z, dj = s->Z;
  size_t c = IX(s, i, j, k), cil = c - di, cjl = c - dj, ckl = c - 1, ciu = c + di, cju = c + dj, cku = c + 1;
  double **NL = s->NL;
  const double dXI = s->p.dxi, dET = s->p.det, dZT = s->p.dzt;
  splitj A = split_at(s, cil, 0), B = split_at(s, cjl, 1), C = split_at(s, ckl, 2);
  double LL1 = (-A.p11 * NL[0][cil] - A.p12 * NL[1][cil] - A.p13 * NL[2][cil] - A.p14 * NL[3][cil]) / dXI +
               (-B.p11 * NL[0][cjl] - B.p12 * NL[1][cjl] - B.p13 * NL[2][cjl] - B.p14 * NL[3][cjl]) / dET +
               (-C.p11 * NL[0][ckl] - C.p12 * NL[1][ckl] - C.p13 * NL[2][ckl] - C.p14 * NL[3][ckl]) / dZT;
  double LL2 = (-A.p21 * NL[0][cil] - A.p22 * NL[1][cil]) / dXI + (-B.p21 * NL[0][cjl] - B.p22 * NL[1][cjl]) / dET +
               (-C.p21 * NL[0][ckl] - C.p22 * NL[1][ckl]) / dZT;
  double LL3 = (-A.p31 * NL[0][cil] - A.p22 * NL[2][cil]) / dXI + (-B.p31 * NL[0][cjl] - B.p22 * NL[2][cjl]) / dET +
               (-C.p31 * NL[0][ckl] - C.p22 * NL[2][ckl]) / dZT;
  double LL4 = (-A.p41 * NL[0][cil] - A.p22 * NL[3][cil]) / dXI + (-B.p41 * NL[0][cjl] - B.p22 * NL[3][cjl]) / dET +
               (-C.p41 * NL[0][ckl] - C.p22 * NL[3][ckl]) / dZT;
  double LL5 =
      (-A.p51 * NL[0][cil] - A.p52 * NL[1][cil] - A.p53 * NL[2][cil] - A.p54 * NL[3][cil] - A.p22 * NL[4][cil]) / dXI +
      (-B.p51 * NL[0][cjl] - B.p52 * NL[1][cjl] - B.p53 * NL[2][cjl] - B.p54 * NL[3][cjl] - B.p22 * NL[4][cjl]) / dET +
      (-C.p51 * NL[0][ckl] - C.p52 * NL[1][ckl] - C.p53 * NL[2][ckl] - C.p54 * NL[3][ckl] - C.p22 * NL[4][ckl]) / dZT;
  A = split_at(s, ciu, 0); B = split_at(s, cju, 1); C = split_at(s, cku, 2);
  double UU1 = (+A.m11 * NL[0][ciu] + A.p12 * NL[1][ciu] + A.p13 * NL[2][ciu] + A.p14 * NL[3][ciu]) / dXI +
               (+B.m11 * NL[0][cju] + B.p12 * NL[1][cju] + B.p13 * NL[2][cju] + B.p14 * NL[3][cju]) / dET +
               (+C.m11 * NL[0][cku] + C.p12 * NL[1][cku] + C.p13 * NL[2][cku] + C.p14 * NL[3][cku]) / dZT;
  double UU2 = (+A.p21 * NL[0][ciu] + A.m22 * NL[1][ciu]) / dXI + (+B.p21 * NL[0][cju] + B.m22 * NL[1][cju]) / dET +
               (+C.p21 * NL[0][cku] + C.m22 * NL[1][cku]) / dZT;
  double UU3 = (+A.p31 * NL[0][ciu] + A.m22 * NL[2][ciu]) / dXI + (+B.p31 * NL[0][cju] + B.m22 * NL[2][cju]) / dET +
               (+C.p31 * NL[0][cku] + C.m22 * NL[2][cku]) / dZT;
  double UU4 = (+A.p41 * NL[0][ciu] + A.m22 * NL[3][ciu]) / dXI + (+B.p41 * NL[0][cju] + B.m22 * NL[3][cju]) / dET +
               (+C.p41 * NL[0][cku] + C.m22 * NL[3][cku]) / dZT;
  double UU5 =
      (+A.p51 * NL[0][ciu] + A.p52 * NL[1][ciu] + A.p53 * NL[2][ciu] + A.p54 * NL[3][ciu] + A.m22 * NL[4][ciu]) / dXI +
      (+B.p51 * NL[0][cju] + B.p52 * NL[1][cju] + B.p53 * NL[2][cju] + B.p54 * NL[3][cju] + B.m22 * NL[4][cju]) / dET +
      (+C.p51 * NL[0][cku] + C.p52 * NL[1][cku] + C.p53 * NL[2][cku] + C.p54 * NL[3][cku] + C.m22 * NL[4][cku]) / dZT;
  cprim q = cp_at(s, c);
  diag3 d = diag_at(s, c, &q);
  double **MR = s->MR, **NR = s->NR;
  NR[0][c] = d.d11 * (MR[0][c] - LL1 - UU1);
  NR[1][c] = d.d22 * (MR[1][c] - LL2 - UU2);
  NR[2][c] = d.d22 * (MR[2][c] - LL3 - UU3);
  NR[3][c] = d.d22 * (MR[3][c] - LL4 - UU4);
  NR[4][c] = d.d51 * (MR[0][c] - LL1 - UU1) + d.d22 * (MR[4][c] - LL5 - UU5);
}

/* four Jacobi relaxations, DPLUSGS.cpp:488-1141; before each one the
 * periodic 1-plane x halo of NL (NL[2] <- NL[ie], NL[ie+1] <- NL[3], the
 * self-copies of :510-531), after it NL <- NR on the interior (:1127-1139).
 * NL starts as D^-1 MR with zero ghost rows, as or_dts_residual leaves it
 * (:186-478 form the same values: the sponge terms that Dual_time_stepping
 * adds are zero here). */
void or_dplur_sweeps(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  const size_t plane = (size_t)s->Y * s->Z;
  for (int sweep = 1; sweep <= 4; sweep++) {
    for (int v = 0; v < 5 && !s->p.x_open; v++) {   /* open: the end planes stay zero */
      memmove(s->NL[v] + 2 * plane, s->NL[v] + (size_t)ie * plane, plane * sizeof(double));
      memmove(s->NL[v] + (size_t)(ie + 1) * plane, s->NL[v] + 3 * plane, plane * sizeof(double));
    }
    for (int i = 3; i <= ie; i++)
      for (int j = 2; j <= jn; j++)
        for (int k = 2; k <= kn; k++) dplur_cell(s, i, j, k);
    for (int i = 3; i <= ie; i++)
      for (int j = 2; j <= jn; j++)
        for (int k = 2; k <= kn; k++) {
          size_t c = IX(s, i, j, k);
          for (int v = 0; v < 5; v++) s->NL[v][c] = s->NR[v][c];
        }
  }
}

/* primitive-variable update of DPLUSGS.cpp:1152-1196 (as or_update, but the
 * first increment is that of the pressure) and its norms, :1203-1221:
 * er[v] = sqrt(sum of the squared squared increments) / (Nx Ny Nz) */
void or_dplur_update(or_state *s, double *er) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  double e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        const double J = s->J[c];
        double **q = s->U_, **NR = s->NR;
        double rhoold = q[0][c] * J;
        double Uold = q[1][c] / q[0][c];
        double Vold = q[2][c] / q[0][c];
        double Wold = q[3][c] / q[0][c];
        double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
        double Pold = (q[4][c] * J - 0.5 * rhoold * VVold) * (KG - 1);
        double Told = Pold / rhoold;
        double P = Pold + NR[0][c] * J;
        double U = Uold + NR[1][c] * J;
        double V = Vold + NR[2][c] * J;
        double W = Wold + NR[3][c] * J;
        double T = Told + NR[4][c] * J;
        double rho = P / T;
        q[0][c] = rho / J;
        q[1][c] = rho * U / J;
        q[2][c] = rho * V / J;
        q[3][c] = rho * W / J;
        q[4][c] = (P / (KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / J;
        s->res[0][c] = (P - Pold) * (P - Pold);
        s->res[1][c] = (U - Uold) * (U - Uold);
        s->res[2][c] = (V - Vold) * (V - Vold);
        s->res[3][c] = (W - Wold) * (W - Wold);
        s->res[4][c] = (T - Told) * (T - Told);
      }
  /* the sums run in a second pass in the reference's loop order (:1203-1215) */
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        e1 = e1 + s->res[0][c] * s->res[0][c];
        e2 = e2 + s->res[1][c] * s->res[1][c];
        e3 = e3 + s->res[2][c] * s->res[2][c];
        e4 = e4 + s->res[3][c] * s->res[3][c];
        e5 = e5 + s->res[4][c] * s->res[4][c];
      }
  double DN = 1. / ((double)s->p.nx * s->p.ny * s->p.nz);
  er[0] = sqrt(e1) * DN; er[1] = sqrt(e2) * DN; er[2] = sqrt(e3) * DN;
  er[3] = sqrt(e4) * DN; er[4] = sqrt(e5) * DN;
}

/* one inner iteration with DPLUSGS in place of Dual_time_stepping */
void or_dplur_inner_iteration(or_state *s, double *er) {
  or_halo_x(s);
  or_bc_y(s);
  or_bc_x(s);
  or_bc_z(s);
  or_flux_x(s);
  or_flux_y(s);
  or_flux_z(s);
  or_viscous(s);
  or_dplur_residual(s);
  or_dplur_sweeps(s);
  or_dplur_update(s, er);
}

/* one inner iteration: main.cpp:167-264 */
void or_inner_iteration(or_state *s, double *er) {
  or_halo_x(s);
  or_bc_y(s);
  or_bc_x(s);
  or_bc_z(s);
  or_flux_x(s);
  or_flux_y(s);
  or_flux_z(s);
  or_viscous(s);
  or_dts_residual(s);
  or_sweeps(s);
  or_update(s, er);
}

/* bulk mass flux with the weighting of Driven_force.cpp:38-62 */
double or_bulk_flux(or_state *s) {
  const int ie = s->p.nx + 2, jn = s->p.ny + 1, kn = s->p.nz + 1;
  double Jsum = 0;
  for (int j = 2; j <= jn; j++) Jsum = Jsum + 1. / s->J[IX(s, 3, j, 3)];
  double Q = 0, temp;
  for (int i = 3; i <= ie; i++)
    for (int j = 2; j <= jn; j++)
      for (int k = 2; k <= kn; k++) {
        size_t c = IX(s, i, j, k);
        temp = (s->U_[1][c] * s->J[c]) * 1. / s->J[c] / Jsum;
        Q = Q + temp;
      }
  return Q / s->p.nx / s->p.nz;
}

/* time-level shift, main.cpp:364-386 */
void or_end_step(or_state *s) {
  const int ie = s->p.nx + 2;
  size_t plane = (size_t)s->Y * s->Z;
  for (int v = 0; v < 5; v++) {
    size_t off = 2 * plane, len = (size_t)ie * plane;   /* planes 2..gend+1 */
    memmove(s->Uq[v] + off, s->U[v] + off, len * sizeof(double));
    memmove(s->U[v] + off, s->U_[v] + off, len * sizeof(double));
  }
}
