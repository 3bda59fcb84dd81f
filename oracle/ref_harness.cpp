/*
 * Test-infrastructure harness around the reference's own hot-path routines.
 *
 * Compiled by oracle/build_ref.py together with the reference sources (taken
 * from the reference tree at build time, patched in memory, never copied)
 * into oracle/_ref/<config>/libref.so.  It plays the part of the reference's
 * main.cpp: it owns the arrays that Array.h would allocate, runs the set-up
 * calls of main.cpp:90-141 and exposes the body of the inner-iteration loop
 * (main.cpp:157-264) and the end-of-step block (main.cpp:304-386) as C
 * entry points so tests can drive it step by step and read any array back.
 *
 * The grid sizes are compile-time constants of the generated Resolution.h,
 * exactly as in the reference; one library is built per configuration.
 * The run is a single process.  For the periodic channel the MPI stub
 * presents it as rank 1 of 3 (CGLI_MYID 1, CGLI_NSLAB 3), which makes every
 * routine take its interior path and turns the x halos into periodic
 * self-copies (see mpi_stub/mpi.h); for the open (inflow/outflow)
 * configuration as rank 0 of 1, which takes every first- and last-rank
 * branch.
 */
#include <mpi.h>
#include <omp.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Resolution.h"

int cgli_stub_rank = CGLI_MYID;
int cgli_stub_size = CGLI_NSLAB;
char cgli_stub_initial_path[4096];
/* values the patched body-force line of Dual_time_stepping.cpp:831 reads:
 * the reference's buoyancy when cgli_ref_buoyancy, else the uniform force */
double cgli_ref_force = 0.0;
int cgli_ref_buoyancy = 0;
int X_np;

typedef double (*A3)[Y_m][Z_m];

/* prototypes of the reference routines, as declared in main.h:164-986 */
void Jacobian(int, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Jacobian_u(int, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Jacobian_v(int, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Jacobian_w(int, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Initial_condition(int, int, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Y_boundary_condition(int, double, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                          A3, A3, A3, A3, A3, A3, A3);
void X_boundary_condition(int, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                          A3, A3, A3, A3, A3, A3);
void Z_boundary_condition(int, A3, A3, A3, A3, A3, A3);
void Flux_X(int, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
            A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Flux_Y(int, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
            A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Flux_Z(int, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
            A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Viscous_terms(int, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                   A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Dual_time_stepping(int, double, double, double *, double *, double *, double *, double *,
                        int (*)[2], int (*)[3],
                        A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                        A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                        A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                        A3, A3, A3, A3,
                        A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
                        A3, A3, A3, A3, A3, A3, A3);
void DPLUSGS(int, double, double *, double *, double *, double *, double *, double,
             A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
             A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
             A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
             A3, A3, A3, A3,
             A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
             A3, A3, A3, A3, A3);
void Driven_force(int, A3, A3);
void Hyperplane(int, int (*)[2], int (*)[3]);
void Filter(int, double, double, double, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);
void Statistic(int, int, int, int, double, double, double, double, double, double,
               A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3,
               A3, A3, A3, A3, A3, A3, A3, A3, A3, A3, A3);

namespace {

const int MYID = CGLI_MYID;

struct Arrays {
  A3 U_[5], U[5], Uq[5];
  A3 J, m[9];
  A3 Ju, mu[9], Jv, mv[9], Jw, mw[9];
  A3 inFx[5], inFy[5], inFz[5], vF[4];
  A3 MR[5], ML[5], NR[5], NL[5], LR[5], LL[5], Res[5];
  A3 EpX, EpY, EpZ, Xp, Yp, Zp;
  int (*Nijk)[2];
  int (*ijk)[3];
  int nplane_rows, ncell_rows;
};

Arrays A;
bool allocated = false;
double g_dt = 0.0, g_e = 1e-4;

int gend1() { return (X_out / CGLI_NSLAB) + 2; } /* gend[MYID] of Mpi_division.h */

A3 alloc3() {
  /* value-initialised, unlike Array.h:7-186 (patch P10) */
  return (A3)calloc((size_t)X_np * Y_m * Z_m, sizeof(double));
}

struct Named { const char *name; A3 *slot; };

}  // namespace

extern "C" {

int ref_dims(int *out) {
  out[0] = X_out / CGLI_NSLAB; out[1] = Y_out; out[2] = Z_out;
  out[3] = X_out / CGLI_NSLAB + 6; out[4] = Y_m; out[5] = Z_m;
  return 0;
}

void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

/* builds the i+j+k hyperplane lists with the same order as Hyperplane.cpp:50-78
 * (m ascending, then i, j, k ascending) in O(N) instead of O(N * planes) */
static void build_hyperplanes_fast() {
  int iend = gend1();
  int ii = 0;
  for (int m = 7; m <= iend + ny + nz; m++) {
    int mi = 0;
    for (int i = 3; i <= iend; i++)
      for (int j = 2; j < nyy; j++) {
        int k = m - i - j;
        if (k >= 2 && k < nzz) {
          ii++; mi++;
          A.ijk[ii][0] = i; A.ijk[ii][1] = j; A.ijk[ii][2] = k;
        }
      }
    A.Nijk[m][0] = ii;
    A.Nijk[m][1] = mi;
  }
}

/* runs the reference Hyperplane() into fresh lists and compares with the fast
 * enumeration; returns the number of mismatching entries */
long ref_check_hyperplanes() {
  int (*N2)[2] = (int (*)[2])calloc((size_t)((X_np - 3) + ny + nz + 7), sizeof(int[2]));
  int (*c2)[3] = (int (*)[3])calloc((size_t)(X_np - 6) * Y_out * Z_out * 3, sizeof(int[3]));
  Hyperplane(MYID, N2, c2);
  long bad = 0;
  int iend = gend1();
  for (int m = 7; m <= iend + ny + nz; m++) {
    if (N2[m][0] != A.Nijk[m][0] || N2[m][1] != A.Nijk[m][1]) bad++;
  }
  long n = (long)(X_out / CGLI_NSLAB) * Y_out * Z_out;
  for (long t = 1; t <= n; t++)
    for (int d = 0; d < 3; d++) if (c2[t][d] != A.ijk[t][d]) bad++;
  free(N2); free(c2);
  return bad;
}

/* main.cpp:87-141: allocation, metrics, hyperplanes, initial condition read
 * from a restart file in the layout of Initial_condition.cpp:136-221 */
/* arrays, hyperplane lists and the reference's metrics */
int ref_setup(double deltaT, double e) {
  X_np = X_out / CGLI_NSLAB + 6;
  if (!allocated) {
    for (int v = 0; v < 5; v++) {
      A.U_[v] = alloc3(); A.U[v] = alloc3(); A.Uq[v] = alloc3();
      A.inFx[v] = alloc3(); A.inFy[v] = alloc3(); A.inFz[v] = alloc3();
      A.MR[v] = alloc3(); A.ML[v] = alloc3(); A.NR[v] = alloc3(); A.NL[v] = alloc3();
      A.LR[v] = alloc3(); A.LL[v] = alloc3(); A.Res[v] = alloc3();
    }
    for (int v = 0; v < 4; v++) A.vF[v] = alloc3();
    A.J = alloc3(); A.Ju = alloc3(); A.Jv = alloc3(); A.Jw = alloc3();
    for (int v = 0; v < 9; v++) { A.m[v] = alloc3(); A.mu[v] = alloc3(); A.mv[v] = alloc3(); A.mw[v] = alloc3(); }
    A.EpX = alloc3(); A.EpY = alloc3(); A.EpZ = alloc3();
    A.Xp = alloc3(); A.Yp = alloc3(); A.Zp = alloc3();
    A.Nijk = (int (*)[2])calloc((size_t)((X_np - 3) + ny + nz + 7), sizeof(int[2]));
    A.ijk = (int (*)[3])calloc((size_t)(X_np - 6) * Y_out * Z_out + 2, sizeof(int[3]));
    allocated = true;
  }
  g_dt = deltaT; g_e = e;
  build_hyperplanes_fast();
  A3 *m = A.m, *mu = A.mu, *mv = A.mv, *mw = A.mw;
  Jacobian(MYID, A.J, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
  Jacobian_u(MYID, A.Ju, mu[0], mu[1], mu[2], mu[3], mu[4], mu[5], mu[6], mu[7], mu[8]);
  Jacobian_v(MYID, A.Jv, mv[0], mv[1], mv[2], mv[3], mv[4], mv[5], mv[6], mv[7], mv[8],
             A.J, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
  Jacobian_w(MYID, A.Jw, mw[0], mw[1], mw[2], mw[3], mw[4], mw[5], mw[6], mw[7], mw[8]);
  return 0;
}

/* the initial field through the reference's restart reader (uses J) */
int ref_load(const char *initial_path) {
  int sw = 0;
  if (initial_path && initial_path[0]) {
    strncpy(cgli_stub_initial_path, initial_path, sizeof(cgli_stub_initial_path) - 1);
    sw = 1;
  }
  Initial_condition(MYID, sw, A.U_[0], A.U_[1], A.U_[2], A.U_[3], A.U_[4],
                    A.U[0], A.U[1], A.U[2], A.U[3], A.U[4],
                    A.Uq[0], A.Uq[1], A.Uq[2], A.Uq[3], A.Uq[4], A.J);
  /* main.cpp:127-141 */
  for (int i = 3; i <= gend1(); i++)
    for (int j = 2; j < nyy; j++)
      for (int k = 2; k < nzz; k++)
        for (int v = 0; v < 5; v++) A.U_[v][i][j][k] = A.U[v][i][j][k];
  return 0;
}

int ref_init(const char *initial_path, double deltaT, double e) {
  ref_setup(deltaT, e);
  return ref_load(initial_path);
}

void ref_set_force(double f) { cgli_ref_force = f; }
void ref_set_buoyancy(int on) { cgli_ref_buoyancy = on; }
double ref_get_force(void) { return cgli_ref_force; }

double *ref_array(const char *name) {
  static char buf[64];
  const Named table[] = {
    {"U1_", &A.U_[0]}, {"U2_", &A.U_[1]}, {"U3_", &A.U_[2]}, {"U4_", &A.U_[3]}, {"U5_", &A.U_[4]},
    {"U1", &A.U[0]}, {"U2", &A.U[1]}, {"U3", &A.U[2]}, {"U4", &A.U[3]}, {"U5", &A.U[4]},
    {"U1q", &A.Uq[0]}, {"U2q", &A.Uq[1]}, {"U3q", &A.Uq[2]}, {"U4q", &A.Uq[3]}, {"U5q", &A.Uq[4]},
    {"J", &A.J}, {"J_u", &A.Ju}, {"J_v", &A.Jv}, {"J_w", &A.Jw},
    {"EpX", &A.EpX}, {"EpY", &A.EpY}, {"EpZ", &A.EpZ}, {"Y_point", &A.Yp},
  };
  for (const Named &n : table) if (strcmp(n.name, name) == 0) return (double *)*n.slot;
  const char *mnames[9] = {"xidx", "xidy", "xidz", "etdx", "etdy", "etdz", "ztdx", "ztdy", "ztdz"};
  for (int v = 0; v < 9; v++) {
    if (strcmp(name, mnames[v]) == 0) return (double *)A.m[v];
    snprintf(buf, sizeof buf, "%s_u", mnames[v]); if (strcmp(name, buf) == 0) return (double *)A.mu[v];
    snprintf(buf, sizeof buf, "%s_v", mnames[v]); if (strcmp(name, buf) == 0) return (double *)A.mv[v];
    snprintf(buf, sizeof buf, "%s_w", mnames[v]); if (strcmp(name, buf) == 0) return (double *)A.mw[v];
  }
  struct { const char *pfx; A3 *arr; int n; int base; } groups[] = {
    {"inFx", A.inFx, 5, 1}, {"inFy", A.inFy, 5, 1}, {"inFz", A.inFz, 5, 1}, {"vF", A.vF, 4, 2},
    {"MR", A.MR, 5, 1}, {"ML", A.ML, 5, 1}, {"NR", A.NR, 5, 1}, {"NL", A.NL, 5, 1},
    {"LR", A.LR, 5, 1}, {"LL", A.LL, 5, 1}, {"Residual", A.Res, 5, 1},
  };
  for (auto &g : groups)
    for (int v = 0; v < g.n; v++) {
      snprintf(buf, sizeof buf, "%s%d", g.pfx, v + g.base);
      if (strcmp(name, buf) == 0) return (double *)g.arr[v];
    }
  return nullptr;
}

/* main.cpp:167-210: periodic Q halo (the stub's self-copy Sendrecv), then the
 * Y, X and Z boundary routines in the reference's order */
void ref_halo_bc(void) {
  int istart = 3, iend = gend1();
  int l_nbr = MYID == 0 ? MPI_PROC_NULL : MYID - 1;
  int r_nbr = MYID == CGLI_NSLAB - 1 ? MPI_PROC_NULL : MYID + 1;
  int icount = 3 * Y_m * Z_m;
  MPI_Status st[8];
  for (int v = 0; v < 5; v++)
    MPI_Sendrecv((void *)&A.U_[v][istart][0][0], icount, MPI_DOUBLE, l_nbr, 110,
                 (void *)&A.U_[v][iend + 1][0][0], icount, MPI_DOUBLE, r_nbr, 110, MPI_COMM_WORLD, st);
  for (int v = 0; v < 5; v++)
    MPI_Sendrecv((void *)&A.U_[v][iend - 2][0][0], icount, MPI_DOUBLE, r_nbr, 160,
                 (void *)&A.U_[v][istart - 3][0][0], icount, MPI_DOUBLE, l_nbr, 160, MPI_COMM_WORLD, st);
  A3 *q = A.U_, *u = A.U, *uq = A.Uq;
  Y_boundary_condition(MYID, g_dt, g_e, 104.0, q[0], q[1], q[2], q[3], q[4], u[0], u[1], u[2], u[3], u[4],
                       uq[0], uq[1], uq[2], uq[3], uq[4], A.m[4], A.J);
  X_boundary_condition(MYID, g_dt, g_e, q[0], q[1], q[2], q[3], q[4], u[0], u[1], u[2], u[3], u[4],
                       uq[0], uq[1], uq[2], uq[3], uq[4], A.J);
  Z_boundary_condition(MYID, q[0], q[1], q[2], q[3], q[4], A.J);
}

void ref_flux_x(void) {
  A3 *q = A.U_, *mu = A.mu;
  Flux_X(MYID, 1.0, g_e, q[0], q[1], q[2], q[3], q[4], A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4],
         A.ML[0], A.ML[1], A.ML[2], A.ML[3], A.ML[4], A.J, A.Ju,
         mu[0], mu[1], mu[2], mu[3], mu[4], mu[5], mu[6], mu[7], mu[8],
         A.inFx[0], A.inFx[1], A.inFx[2], A.inFx[3], A.inFx[4], A.EpX);
}
void ref_flux_y(void) {
  A3 *q = A.U_, *mv = A.mv;
  Flux_Y(MYID, 1.0, g_e, q[0], q[1], q[2], q[3], q[4], A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4],
         A.ML[0], A.ML[1], A.ML[2], A.ML[3], A.ML[4], A.J, A.Jv,
         mv[0], mv[1], mv[2], mv[3], mv[4], mv[5], mv[6], mv[7], mv[8],
         A.inFy[0], A.inFy[1], A.inFy[2], A.inFy[3], A.inFy[4], A.EpY);
}
void ref_flux_z(void) {
  A3 *q = A.U_, *mw = A.mw;
  Flux_Z(MYID, 1.0, g_e, q[0], q[1], q[2], q[3], q[4], A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4],
         A.ML[0], A.ML[1], A.ML[2], A.ML[3], A.ML[4], A.J, A.Jw,
         mw[0], mw[1], mw[2], mw[3], mw[4], mw[5], mw[6], mw[7], mw[8],
         A.inFz[0], A.inFz[1], A.inFz[2], A.inFz[3], A.inFz[4], A.EpZ);
}
void ref_viscous(void) {
  A3 *q = A.U_, *m = A.m, *mu = A.mu, *mv = A.mv, *mw = A.mw;
  Viscous_terms(MYID, q[0], q[1], q[2], q[3], q[4], A.vF[0], A.vF[1], A.vF[2], A.vF[3],
                A.J, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8],
                A.Ju, mu[0], mu[1], mu[2], mu[3], mu[4], mu[5], mu[6], mu[7], mu[8],
                A.Jv, mv[0], mv[1], mv[2], mv[3], mv[4], mv[5], mv[6], mv[7], mv[8],
                A.Jw, mw[0], mw[1], mw[2], mw[3], mw[4], mw[5], mw[6], mw[7], mw[8],
                A.LR[0], A.LR[1], A.LR[2], A.LR[3], A.LR[4], A.LL[0], A.LL[1], A.LL[2], A.LL[3], A.LL[4],
                A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4], A.ML[0], A.ML[1], A.ML[2], A.ML[3], A.ML[4],
                A.NR[0], A.NR[1], A.NR[2], A.NR[3], A.NR[4], A.NL[0], A.NL[1], A.NL[2], A.NL[3], A.NL[4]);
}
void ref_dts(double *er) {
  A3 *q = A.U_, *u = A.U, *uq = A.Uq, *m = A.m;
  Dual_time_stepping(MYID, g_dt, g_e, &er[0], &er[1], &er[2], &er[3], &er[4], A.Nijk, A.ijk,
                     q[0], q[1], q[2], q[3], q[4], u[0], u[1], u[2], u[3], u[4],
                     uq[0], uq[1], uq[2], uq[3], uq[4],
                     A.J, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8],
                     A.inFx[0], A.inFx[1], A.inFx[2], A.inFx[3], A.inFx[4],
                     A.inFy[0], A.inFy[1], A.inFy[2], A.inFy[3], A.inFy[4],
                     A.inFz[0], A.inFz[1], A.inFz[2], A.inFz[3], A.inFz[4],
                     A.vF[0], A.vF[1], A.vF[2], A.vF[3],
                     A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4],
                     A.NR[0], A.NR[1], A.NR[2], A.NR[3], A.NR[4],
                     A.NL[0], A.NL[1], A.NL[2], A.NL[3], A.NL[4],
                     A.Res[0], A.Res[1], A.Res[2], A.Res[3], A.Res[4], A.mv[4], A.Jv);
}

/* one pass of the body of the inner loop, main.cpp:167-264 */
void ref_inner_iteration(double *er) {
  ref_halo_bc();
  ref_flux_x();
  ref_flux_y();
  ref_flux_z();
  ref_viscous();
  ref_dts(er);
}

/* DPLUSGS.cpp in place of Dual_time_stepping (the call main.cpp:268-284
 * leaves commented out): residual, four Jacobi relaxations, update */
void ref_dplusgs(double *er) {
  A3 *q = A.U_, *u = A.U, *uq = A.Uq, *m = A.m;
  DPLUSGS(MYID, g_dt, &er[0], &er[1], &er[2], &er[3], &er[4], g_e,
          q[0], q[1], q[2], q[3], q[4], u[0], u[1], u[2], u[3], u[4],
          uq[0], uq[1], uq[2], uq[3], uq[4],
          A.J, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8],
          A.inFx[0], A.inFx[1], A.inFx[2], A.inFx[3], A.inFx[4],
          A.inFy[0], A.inFy[1], A.inFy[2], A.inFy[3], A.inFy[4],
          A.inFz[0], A.inFz[1], A.inFz[2], A.inFz[3], A.inFz[4],
          A.vF[0], A.vF[1], A.vF[2], A.vF[3],
          A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4],
          A.NR[0], A.NR[1], A.NR[2], A.NR[3], A.NR[4],
          A.NL[0], A.NL[1], A.NL[2], A.NL[3], A.NL[4],
          A.Res[0], A.Res[1], A.Res[2], A.Res[3], A.Res[4]);
}

void ref_inner_iteration_dplusgs(double *er) {
  ref_halo_bc();
  ref_flux_x();
  ref_flux_y();
  ref_flux_z();
  ref_viscous();
  ref_dplusgs(er);
}

/* bulk mass flux with the weighting of Driven_force.cpp:38-62, over the
 * Nx cells this process owns (the reference divides by the global X_out) */
double ref_bulk_flux(void) {
  double Jsum = 0;
  for (int j = 2; j <= ny; j++) Jsum = Jsum + 1. / A.J[3][j][3];
  double Q = 0, temp;
  for (int i = 3; i <= gend1(); i++)
    for (int j = 2; j < nyy; j++)
      for (int k = 2; k < nzz; k++) {
        temp = (A.U_[1][i][j][k] * A.J[i][j][k]) * 1. / A.J[i][j][k] / Jsum;
        Q = Q + temp;
      }
  return Q / (X_out / CGLI_NSLAB) / Z_out;
}

/* end of a physical step, main.cpp:307 and main.cpp:364-386 */
void ref_end_step(void) {
  Driven_force(MYID, A.U[1], A.J);
  int istart = 3, iend = gend1();
#pragma omp parallel for
  for (int i = istart - 1; i <= iend + 1; i++)
    for (int j = 0; j <= nyyy; j++)
      for (int k = 0; k <= nzzz; k++)
        for (int v = 0; v < 5; v++) {
          A.Uq[v][i][j][k] = A.U[v][i][j][k];
          A.U[v][i][j][k] = A.U_[v][i][j][k];
        }
}

/* Filter.cpp (never called by the reference driver): fills EpX/EpY/EpZ */
void ref_filter(double roe_criterion, double e_high, double e_low) {
  A3 *q = A.U_;
  Filter(MYID, roe_criterion, e_high, e_low, q[0], q[1], q[2], q[3], q[4], A.Yp, A.EpX, A.EpY, A.EpZ, A.J);
}

/* Statistic.cpp:12-506 as main.cpp:334-342 calls it after a step: adds U_
 * to the per-(i, j) sums over k; every statistic_step-th step it writes the
 * means of the planes at x positions obs[0..4] to st_obs<n>_<step>.dat in the
 * current directory (Statistic.cpp:120-331) and clears the sums. */
void ref_statistic(int step, int statistic_step, const double *obs) {
  A3 *q = A.U_, *mv = A.mv;
  Statistic(MYID, step, 0, statistic_step, obs[0], obs[1], obs[2], obs[3], obs[4], g_e,
            q[0], q[1], q[2], q[3], q[4], A.J, A.Jv,
            mv[0], mv[1], mv[2], mv[3], mv[4], mv[5], mv[6], mv[7], mv[8],
            A.MR[0], A.MR[1], A.MR[2], A.MR[3], A.MR[4], A.ML[0], A.ML[1], A.ML[2], A.ML[3], A.ML[4], A.EpY);
}

}  // extern "C"
