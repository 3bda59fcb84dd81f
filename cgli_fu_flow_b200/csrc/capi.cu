// extern "C" entry points of include/cgli_fu_flow.h: context lifetime,
// device memory, array transfer, the reference-routine entry points and the
// physical-step driver (the loop of main.cpp:152-420).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <sys/types.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cgli_fu_flow.h"
#include "cgli_dev.cuh"
#include "cgli_filter.h"
#include "cnn.h"
#include "cgli_launch.h"

#include "host_setup.h"

#include <algorithm>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(call)                                                                    \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fail(CGLI_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e));       \
  } while (0)

const char *kMetricNames[9] = {"xidx", "xidy", "xidz", "etdx", "etdy", "etdz", "ztdx", "ztdy", "ztdz"};

}  // namespace

namespace cgli {
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace cgli

struct cgli_ctx {
  cgli_params p;
  cgli::Dev d;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  long long bytes = 0;
  bool have_metrics = false, have_state = false;
  double *h_norms = nullptr;   // pinned, 8 doubles
  double *d_out = nullptr;     // device scratch for norms / bulk flux
  int update_blocks = 0;         // partial sums of the per-row update kernels (routine path, DP-LUR)
  int sweep_update_blocks = 0;   // partial sums of the update after the wavefront passes
  int sweep_tiles = 0;
  cgli::SweepArgs sw;
  bool metrics_checked = false;
  cudaGraphExec_t iter_graph = nullptr;
  cudaGraphExec_t dts_graph = nullptr;
  cudaEvent_t events[8] = {};
  double Emax[5] = {0, 0, 0, 0, 0};   // running maximum of the norms over the run
  int history = 0;                    // completed steps since the state was set
  int predictor = 0;                  // 0 previous level, 1 extrapolation, 2 learned
  int inner_solver = CGLI_LUSGS;      // CGLI_LUSGS or CGLI_DPLUR
  cudaEvent_t sweep_ev[2] = {};       // recorded around the wavefront passes inside the iteration graph
  double sweep_ms = 0;                // their accumulated device time since the last reset
  long long sweep_passes = 0;
  cgli_cnn *cnn = nullptr;            // learned initial guess (not owned)
  std::vector<double> step_norms;     // the five norms of every inner iteration of the last step
  double *stats = nullptr;            // [CGLI_NSTATS][nx][ny] running sums and samples (allocated on first use)
  long long stat_samples = 0;
  cgli::FilterBufs fb;                // allocated on first use of the filter
  bool have_filter = false, have_ypoint = false;
};

namespace {

int alloc(cgli_ctx *c, size_t bytes, void **out) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return fail(CGLI_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(p, 0, bytes);
  if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  c->allocs.push_back(p);
  c->bytes += (long long)bytes;
  *out = p;
  return CGLI_OK;
}

int field(cgli_ctx *c, double **out) {
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z;
  return alloc(c, n * sizeof(double), (void **)out);
}

bool is_filter_name(const char *name) {
  return !strcmp(name, "Y_point") || !strcmp(name, "EpX") || !strcmp(name, "EpY") || !strcmp(name, "EpZ");
}

// the filter's 18 fields: Y_point, EpX/Y/Z, two levels and the high-pass
// sum of 4 variables, E at h and 2h
int ensure_filter(cgli_ctx *c) {
  if (c->have_filter) return CGLI_OK;
  cgli::FilterBufs &b = c->fb;
  int rc = field(c, &b.yp);
  for (int f = 0; f < 3 && !rc; f++) rc = field(c, &b.ep[f]);
  for (int v = 0; v < 4 && !rc; v++) {
    rc = field(c, &b.lev[0][v]);
    if (!rc) rc = field(c, &b.lev[1][v]);
    if (!rc) rc = field(c, &b.acc[v]);
  }
  if (!rc) rc = field(c, &b.eh);
  if (!rc) rc = field(c, &b.e2h);
  if (!rc) c->have_filter = true;
  return rc;
}

// device array of a reference name; *is_metric tells whether it is one of
// the 40 metric arrays
double *lookup(cgli_ctx *c, const char *name, bool *is_metric = nullptr) {
  if (is_metric) *is_metric = false;
  cgli::Dev &d = c->d;
  char buf[32];
  for (int v = 0; v < 5; v++) {
    snprintf(buf, sizeof buf, "U%d_", v + 1); if (!strcmp(name, buf)) return d.U_[v];
    snprintf(buf, sizeof buf, "U%d", v + 1); if (!strcmp(name, buf)) return d.U[v];
    snprintf(buf, sizeof buf, "U%dq", v + 1); if (!strcmp(name, buf)) return d.Uq[v];
    snprintf(buf, sizeof buf, "U%dqq", v + 1); if (!strcmp(name, buf)) return d.Uqq[v];
    snprintf(buf, sizeof buf, "MR%d", v + 1); if (!strcmp(name, buf)) return d.MR[v];
    snprintf(buf, sizeof buf, "NR%d", v + 1); if (!strcmp(name, buf)) return d.NR[v];
    snprintf(buf, sizeof buf, "NL%d", v + 1); if (!strcmp(name, buf)) return d.NL[v];
    snprintf(buf, sizeof buf, "inFx%d", v + 1); if (!strcmp(name, buf)) return d.inF[0][v];
    snprintf(buf, sizeof buf, "inFy%d", v + 1); if (!strcmp(name, buf)) return d.inF[1][v];
    snprintf(buf, sizeof buf, "inFz%d", v + 1); if (!strcmp(name, buf)) return d.inF[2][v];
  }
  for (int v = 0; v < 4; v++) {
    snprintf(buf, sizeof buf, "vF%d", v + 2); if (!strcmp(name, buf)) return d.vF[v];
  }
  if (c->have_filter) {
    if (!strcmp(name, "Y_point")) return c->fb.yp;
    if (!strcmp(name, "EpX")) return c->fb.ep[0];
    if (!strcmp(name, "EpY")) return c->fb.ep[1];
    if (!strcmp(name, "EpZ")) return c->fb.ep[2];
  }
  if (is_metric) *is_metric = true;
  if (!strcmp(name, "J")) return d.J;
  const char *fs[3] = {"_u", "_v", "_w"};
  for (int f = 0; f < 3; f++) {
    snprintf(buf, sizeof buf, "J%s", fs[f]); if (!strcmp(name, buf)) return d.Jf[f];
  }
  for (int v = 0; v < 9; v++) {
    if (!strcmp(name, kMetricNames[v])) return d.m[v];
    for (int f = 0; f < 3; f++) {
      snprintf(buf, sizeof buf, "%s%s", kMetricNames[v], fs[f]); if (!strcmp(name, buf)) return d.mf[f][v];
    }
  }
  return nullptr;
}

int check(cgli_ctx *c) {
  if (!c) return fail(CGLI_EINVAL, "null context");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return CGLI_OK;
}

int check_channel_metrics(cgli_ctx *c);

int need_ready(cgli_ctx *c) {
  if (!c->have_metrics) return fail(CGLI_ESTATE, "metrics not set (cgli_channel_metrics / cgli_set_array)");
  if (!c->have_state) return fail(CGLI_ESTATE, "state not set (cgli_set_state)");
  // quantities derived from the metrics (1/J, the channel tables), once per change
  if (!c->metrics_checked) { int rc = check_channel_metrics(c); if (rc) return rc; }
  return CGLI_OK;
}

int last_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return CGLI_OK;
}

int read_norms(cgli_ctx *c, double er[5], int nblocks) {
  double scale = 1.0 / ((double)c->p.nx * c->p.ny * c->p.nz);
  cgli::launch_norms(c->d, c->stream, nblocks, scale, c->d_out);
  CUDA_TRY(cudaMemcpyAsync(c->h_norms, c->d_out, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  int status = 0;
  CUDA_TRY(cudaMemcpy(&status, c->d.status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status) {
    int zero = 0;
    cudaMemcpy(c->d.status, &zero, sizeof(int), cudaMemcpyHostToDevice);
    return fail(CGLI_ETIMEOUT, "a wavefront tile gave up waiting for its neighbour (bounded spin)");
  }
  for (int v = 0; v < 5; v++) er[v] = c->h_norms[v];
  for (int v = 0; v < 5; v++)
    if (!std::isfinite(er[v])) return fail(CGLI_EDIVERGED, "update norm is not finite");
  return CGLI_OK;
}

void drop_graph(cgli_ctx *c) {
  if (c->iter_graph) { cudaGraphExecDestroy(c->iter_graph); c->iter_graph = nullptr; }
}

// Decides whether the cell metrics are those of a grid uniform in x and z
// (xidx = ztdz = 1, the other off-diagonal terms 0, J and etdy functions of
// j alone) over every cell the sweeps read: planes 2..ie+1, rows 2..jn,
// k = 2..kn.  If so the sweeps read J(j), etdy(j) from two small tables
// instead of ten 3-D arrays.  On an open slab the end planes only enter
// through products with their zero implicit halo, so planes 3..ie decide
// (the end planes' ztdy, ztdz are zero there, Jacobian.cpp:110-157).
int check_channel_metrics(cgli_ctx *c) {
  const cgli::Dev &d = c->d;
  size_t n = (size_t)d.X * d.Y * d.Z;
  std::vector<double> J(n), m[9];
  CUDA_TRY(cudaMemcpy(J.data(), d.J, n * 8, cudaMemcpyDeviceToHost));
  for (int v = 0; v < 9; v++) {
    m[v].resize(n);
    CUDA_TRY(cudaMemcpy(m[v].data(), d.m[v], n * 8, cudaMemcpyDeviceToHost));
  }
  const int ie = d.nx + 2, jn = d.ny + 1, kn = d.nz + 1;
  std::vector<double> jt(d.Y, 0.0), et(d.Y, 0.0);
  bool ok = true;
  for (int j = 2; j <= jn && ok; j++) {
    size_t r = cgli::ix(d, 3, j, 2);
    jt[j] = J[r]; et[j] = m[4][r];
    for (int i = d.x_open ? 3 : 2; i <= (d.x_open ? ie : ie + 1) && ok; i++)
      for (int k = 2; k <= kn && ok; k++) {
        size_t q = cgli::ix(d, i, j, k);
        ok = J[q] == jt[j] && m[4][q] == et[j] && m[0][q] == 1.0 && m[8][q] == 1.0 && m[1][q] == 0.0 &&
             m[2][q] == 0.0 && m[3][q] == 0.0 && m[5][q] == 0.0 && m[6][q] == 0.0 && m[7][q] == 0.0;
      }
  }
  if (ok) {
    CUDA_TRY(cudaMemcpy((void *)c->sw.Jtab, jt.data(), sizeof(double) * d.Y, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy((void *)c->sw.etdytab, et.data(), sizeof(double) * d.Y, cudaMemcpyHostToDevice));
  }
  c->sw.channel_metrics = ok ? 1 : 0;
  c->d.face_tables = 0;
  c->d.face_tables = cgli::check_face_tables(c->d, c->d.status + 8, c->stream) ? 1 : 0;
  cgli::launch_inverse_j(d, c->stream);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->metrics_checked = true;
  drop_graph(c);
  return CGLI_OK;
}

}  // namespace

extern "C" {

const char *cgli_last_error(void) { return g_err.c_str(); }

long long cgli_device_bytes(const cgli_ctx *ctx) { return ctx ? ctx->bytes : 0; }

int cgli_create(const cgli_params *p, cgli_ctx **out) {
  if (!p || !out) return fail(CGLI_EINVAL, "null argument");
  *out = nullptr;
  if (p->nx < 3 || p->ny < 6 || p->nz < 4)
    return fail(CGLI_EINVAL, "grid too small: need Nx >= 3, Ny >= 6, Nz >= 4 (reduced wall stencils)");
  if (p->precision != CGLI_FP64 && p->precision != CGLI_MIXED)
    return fail(CGLI_EINVAL, "precision must be CGLI_FP64 or CGLI_MIXED");
  if (!(p->dxi > 0 && p->det > 0 && p->dzt > 0 && p->dt > 0 && p->e > 0 && p->mu > 0 && p->pr > 0))
    return fail(CGLI_EINVAL, "spacings, time step, e, mu and Pr must be positive");
  if (p->nx_inlet < 0 || p->nx_outlet < 0 || p->nx_inlet + p->nx_outlet > p->nx)
    return fail(CGLI_EINVAL, "sponge layers must satisfy 0 <= nx_inlet, nx_outlet and nx_inlet + nx_outlet <= Nx");
  if (!p->x_open && (p->nx_inlet || p->nx_outlet))
    return fail(CGLI_EINVAL, "sponge layers need x_open (a periodic slab has no inlet or outlet)");
  if ((p->nx_inlet || p->nx_outlet) && !(p->high > 0))
    return fail(CGLI_EINVAL, "sponge layers need the channel height `high` > 0");
  cgli_ctx *c = new cgli_ctx();
  c->p = *p;
  cudaError_t e = cudaGetDevice(&c->device);
  if (e != cudaSuccess) { delete c; return fail(CGLI_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e)); }
  cgli::Dev &d = c->d;
  memset(&d, 0, sizeof d);
  d.nx = p->nx; d.ny = p->ny; d.nz = p->nz;
  d.X = p->nx + 6; d.Y = p->ny + 4; d.Z = p->nz + 4;
  d.dj = d.Z; d.di = (long long)d.Y * d.Z;
  d.dxi = p->dxi; d.det = p->det; d.dzt = p->dzt; d.dt = p->dt; d.e = p->e;
  d.mu = p->mu; d.pr = p->pr; d.twl = p->twall_lo; d.twh = p->twall_hi;
  d.rdxi = 1.0 / p->dxi; d.rdet = 1.0 / p->det; d.rdzt = 1.0 / p->dzt; d.rpr = 1.0 / p->pr;
  d.curved_walls = p->curved_walls ? 1 : 0;
  d.x_open = p->x_open ? 1 : 0;
  d.nx_inlet = p->nx_inlet;
  d.nx_outlet = p->nx_outlet;
  d.buoyancy = p->buoyancy ? 1 : 0;
  d.high = p->high;
  int rc = CGLI_OK;
#define F(x) if (rc == CGLI_OK) rc = field(c, &(x))
  for (int v = 0; v < 5; v++) {
    F(d.U_[v]); F(d.U[v]); F(d.Uq[v]); F(d.Uqq[v]); F(d.MR[v]); F(d.NL[v]); F(d.NR[v]);
    for (int f = 0; f < 3; f++) F(d.inF[f][v]);
  }
  for (int v = 0; v < 4; v++) {
    F(d.vF[v]); F(d.vprim[v]);
    for (int f = 0; f < 3; f++) F(d.vflux[f][v]);
  }
  F(d.J);
  F(d.iJ);
  for (int v = 0; v < 9; v++) F(d.m[v]);
  for (int f = 0; f < 3; f++) {
    F(d.Jf[f]);
    for (int v = 0; v < 9; v++) F(d.mf[f][v]);
  }
#undef F
  if (rc == CGLI_OK) rc = alloc(c, 16 * sizeof(double), (void **)&d.scal);
  if (rc == CGLI_OK) rc = alloc(c, (8 + 296) * sizeof(double), (void **)&c->d_out);
  if (rc == CGLI_OK) rc = alloc(c, 16 * sizeof(int), (void **)&d.status);
  if (rc == CGLI_OK) rc = alloc(c, 3 * 4 * sizeof(double) * d.Y, (void **)&d.ftab);
  c->update_blocks = p->nx * p->ny;
  // the wavefront's tile grid for this context's precision
  const bool mixed_passes = p->precision == CGLI_MIXED;
  const int nti = mixed_passes ? cgli::sweep_tiles_x<float>(p->nx) : cgli::sweep_tiles_x<double>(p->nx);
  const int ntj = mixed_passes ? cgli::sweep_tiles_y<float>(p->ny) : cgli::sweep_tiles_y<double>(p->ny);
  const int tile_i = mixed_passes ? cgli::SweepTile<float>::TI : cgli::SweepTile<double>::TI;
  const int tile_j = mixed_passes ? cgli::SweepTile<float>::TJ : cgli::SweepTile<double>::TJ;
  c->sweep_tiles = nti * ntj;
  c->sweep_update_blocks = cgli::sweep_update_blocks(d, mixed_passes);
  size_t nblk = (size_t)std::max(std::max(c->update_blocks, c->sweep_tiles), c->sweep_update_blocks);
  if (rc == CGLI_OK) rc = alloc(c, 5 * sizeof(double) * nblk, (void **)&d.partial);
  {
    cgli::SweepArgs &a = c->sw;
    memset(&a, 0, sizeof a);
    const bool mixed = p->precision == CGLI_MIXED;
    const size_t es = mixed ? sizeof(float) : sizeof(double);
    const size_t nsk = (size_t)(mixed ? cgli::skew_size<float>(d) : cgli::skew_size<double>(d));
    const size_t plane = (size_t)d.Y * d.Z;
    for (int v = 0; v < 5; v++) {
      if (mixed) {
        if (rc == CGLI_OK) rc = alloc(c, nsk * es, (void **)&a.dqf[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.halo_ff[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.halo_bf[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hxpf[v]);
      } else {
        if (rc == CGLI_OK) rc = alloc(c, nsk * es, (void **)&a.dq[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.halo_f[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.halo_b[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hxp[v]);
      }
    }
    if (rc == CGLI_OK)
      rc = alloc(c, nsk * cgli::CR_N * es, mixed ? (void **)&a.cellrecf : (void **)&a.cellrec);
    for (int v = 0; v < cgli::REC_N; v++) {
      if (mixed) {
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hrecf_f[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hrecf_b[v]);
      } else {
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hrec_f[v]);
        if (rc == CGLI_OK) rc = alloc(c, plane * es, (void **)&a.hrec_b[v]);
      }
    }
    size_t xb = (size_t)c->sweep_tiles * tile_j * p->nz * 5 * es;
    size_t yb = (size_t)c->sweep_tiles * tile_i * p->nz * 5 * es;
    if (rc == CGLI_OK) rc = alloc(c, xb, mixed ? (void **)&a.xbuff : (void **)&a.xbuf);
    if (rc == CGLI_OK) rc = alloc(c, yb, mixed ? (void **)&a.ybuff : (void **)&a.ybuf);
    if (rc == CGLI_OK) rc = alloc(c, 64, (void **)&a.ticket);
    double *jt = nullptr, *et = nullptr;
    if (rc == CGLI_OK) rc = alloc(c, sizeof(double) * d.Y, (void **)&jt);
    if (rc == CGLI_OK) rc = alloc(c, sizeof(double) * d.Y, (void **)&et);
    a.Jtab = jt; a.etdytab = et;
    a.spin_limit = CGLI_WAIT_LIMIT_DEFAULT;
  }
  if (rc == CGLI_OK) {
    cudaError_t e = cgli::sweep_kernel_attributes();
    if (e != cudaSuccess) rc = fail(CGLI_ECUDA, std::string("sweep kernel attributes: ") + cudaGetErrorString(e));
  }
  if (rc == CGLI_OK) {
    // wavefront clusters along x, and the tickets' order of the cluster
    // rows (anti-diagonals of the grid of clusters)
    cgli::SweepArgs &a = c->sw;
    a.cluster_x = cgli::sweep_cluster_x(nti, ntj, mixed_passes);
    std::vector<int> order;
    cgli::sweep_tile_order(nti / a.cluster_x, ntj, order);
    int *dorder = nullptr;
    rc = alloc(c, sizeof(int) * order.size(), (void **)&dorder);
    if (rc == CGLI_OK) cudaMemcpy(dorder, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice);
    a.order = dorder;
  }
  if (rc == CGLI_OK && cudaMallocHost(&c->h_norms, 16 * sizeof(double)) != cudaSuccess)
    rc = fail(CGLI_ENOMEM, "cudaMallocHost");
  if (rc == CGLI_OK && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = fail(CGLI_ECUDA, "cudaStreamCreate");
  if (rc != CGLI_OK) {
    std::string keep = g_err;
    cgli_destroy(c);
    g_err = keep;
    return rc;
  }
  for (auto &e : c->events)
    if (rc == CGLI_OK && cudaEventCreate(&e) != cudaSuccess) rc = fail(CGLI_ECUDA, "cudaEventCreate");
  for (auto &e : c->sweep_ev)
    if (rc == CGLI_OK && cudaEventCreate(&e) != cudaSuccess) rc = fail(CGLI_ECUDA, "cudaEventCreate");
  if (rc != CGLI_OK) {
    std::string keep = g_err;
    cgli_destroy(c);
    g_err = keep;
    return rc;
  }
  double f = p->force;
  cudaMemcpy(d.scal, &f, sizeof f, cudaMemcpyHostToDevice);
  *out = c;
  return CGLI_OK;
}

int cgli_destroy(cgli_ctx *c) {
  if (!c) return CGLI_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->iter_graph) cudaGraphExecDestroy(c->iter_graph);
  if (c->dts_graph) cudaGraphExecDestroy(c->dts_graph);
  for (auto &e : c->events)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->sweep_ev)
    if (e) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  if (c->h_norms) cudaFreeHost(c->h_norms);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return CGLI_OK;
}

int cgli_set_array(cgli_ctx *c, const char *name, const double *host) {
  int rc = check(c); if (rc) return rc;
  if (!name || !host) return fail(CGLI_EINVAL, "null argument");
  if (is_filter_name(name)) { rc = ensure_filter(c); if (rc) return rc; }
  bool is_metric = false;
  double *dst = lookup(c, name, &is_metric);
  if (!dst) return fail(CGLI_EINVAL, std::string("unknown array ") + name);
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z;
  CUDA_TRY(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (is_metric) { c->have_metrics = true; c->metrics_checked = false; c->sw.channel_metrics = 0; drop_graph(c); }
  if (!strcmp(name, "Y_point")) c->have_ypoint = true;
  return CGLI_OK;
}

int cgli_get_array(cgli_ctx *c, const char *name, double *host) {
  int rc = check(c); if (rc) return rc;
  if (!name || !host) return fail(CGLI_EINVAL, "null argument");
  if (is_filter_name(name)) { rc = ensure_filter(c); if (rc) return rc; }
  double *src = lookup(c, name);
  if (!src) return fail(CGLI_EINVAL, std::string("unknown array ") + name);
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z;
  CUDA_TRY(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

static int upload_metrics(cgli_ctx *c, const cgli::MetricSet &M);

int cgli_channel_metrics(cgli_ctx *c, double high, double stretch) {
  int rc = check(c); if (rc) return rc;
  if (!(high > 0 && stretch > 0)) return fail(CGLI_EINVAL, "high and stretch must be positive");
  cgli::MetricSet M;
  cgli::channel_metrics(c->p.nx, c->p.ny, c->p.nz, c->p.det, high, stretch, M, c->p.x_open != 0);
  return upload_metrics(c, M);
}

int cgli_wavy_channel_metrics(cgli_ctx *c, double high, double stretch, double amplitude) {
  int rc = check(c); if (rc) return rc;
  if (c->p.x_open) return fail(CGLI_EINVAL, "the wavy-wall metrics are defined for the periodic slab only");
  if (!(high > 0 && stretch > 0) || !(fabs(amplitude) < 0.5 * high))
    return fail(CGLI_EINVAL, "need high, stretch > 0 and |amplitude| < high / 2");
  cgli::MetricSet M;
  cgli::wavy_metrics(c->p.nx, c->p.ny, c->p.nz, c->p.dxi, c->p.det, high, stretch, amplitude, M);
  return upload_metrics(c, M);
}

static int upload_metrics(cgli_ctx *c, const cgli::MetricSet &M) {
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z;
  CUDA_TRY(cudaMemcpyAsync(c->d.J, M.J.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  for (int v = 0; v < 9; v++) CUDA_TRY(cudaMemcpyAsync(c->d.m[v], M.m[v].data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  for (int f = 0; f < 3; f++) {
    CUDA_TRY(cudaMemcpyAsync(c->d.Jf[f], M.Jf[f].data(), n * 8, cudaMemcpyHostToDevice, c->stream));
    for (int v = 0; v < 9; v++)
      CUDA_TRY(cudaMemcpyAsync(c->d.mf[f][v], M.mf[f][v].data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->have_metrics = true;
  c->metrics_checked = false;
  drop_graph(c);
  return CGLI_OK;
}

int cgli_set_state(cgli_ctx *c, const double *const U_[5], const double *const U[5], const double *const Uq[5]) {
  int rc = check(c); if (rc) return rc;
  if (!U_ || !U || !Uq) return fail(CGLI_EINVAL, "null argument");
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z * sizeof(double);
  for (int v = 0; v < 5; v++) {
    if (!U_[v] || !U[v] || !Uq[v]) return fail(CGLI_EINVAL, "null state array");
    CUDA_TRY(cudaMemcpyAsync(c->d.U_[v], U_[v], n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.U[v], U[v], n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.Uq[v], Uq[v], n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.Uqq[v], Uq[v], n, cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->have_state = true;
  c->history = 0;
  for (double &e : c->Emax) e = 0;
  return CGLI_OK;
}

int cgli_set_levels(cgli_ctx *c, const double *const U[5], const double *const Uq[5]) {
  int rc = check(c); if (rc) return rc;
  if (!U || !Uq) return fail(CGLI_EINVAL, "null argument");
  if (!c->have_state) return fail(CGLI_ESTATE, "state not set (cgli_set_state once before cgli_set_levels)");
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z * sizeof(double);
  for (int v = 0; v < 5; v++) {
    if (!U[v] || !Uq[v]) return fail(CGLI_EINVAL, "null state array");
    CUDA_TRY(cudaMemcpyAsync(c->d.Uqq[v], c->d.Uq[v], n, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.U[v], U[v], n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.U_[v], c->d.U[v], n, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d.Uq[v], Uq[v], n, cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

int cgli_copy_state(cgli_ctx *dst, const cgli_ctx *src) {
  int rc = check(dst); if (rc) return rc;
  if (!src || !src->have_state) return fail(CGLI_ESTATE, "source context has no state");
  if (src->p.nx != dst->p.nx || src->p.ny != dst->p.ny || src->p.nz != dst->p.nz)
    return fail(CGLI_EINVAL, "contexts of different grids");
  CUDA_TRY(cudaStreamSynchronize(src->stream));
  size_t n = (size_t)dst->d.X * dst->d.Y * dst->d.Z * sizeof(double);
  for (int v = 0; v < 5; v++) {
    CUDA_TRY(cudaMemcpyAsync(dst->d.U_[v], src->d.U_[v], n, cudaMemcpyDeviceToDevice, dst->stream));
    CUDA_TRY(cudaMemcpyAsync(dst->d.U[v], src->d.U[v], n, cudaMemcpyDeviceToDevice, dst->stream));
    CUDA_TRY(cudaMemcpyAsync(dst->d.Uq[v], src->d.Uq[v], n, cudaMemcpyDeviceToDevice, dst->stream));
    CUDA_TRY(cudaMemcpyAsync(dst->d.Uqq[v], src->d.Uqq[v], n, cudaMemcpyDeviceToDevice, dst->stream));
  }
  dst->p.force = src->p.force;
  CUDA_TRY(cudaMemcpyAsync(dst->d.scal, &dst->p.force, sizeof(double), cudaMemcpyHostToDevice, dst->stream));
  CUDA_TRY(cudaStreamSynchronize(dst->stream));
  for (int v = 0; v < 5; v++) dst->Emax[v] = src->Emax[v];
  dst->history = src->history;
  dst->have_state = true;
  return CGLI_OK;
}

// ---------------------------------------------------------------- restart
// Field f (0..4: Q^n = U*J, 5..9: Q^(n-1) = Uq*J) of the slab occupies
// [x_offset, x_offset + Nx) of a global x extent, k fastest: the MPI-IO
// layout of Output.cpp:187-284 / Initial_condition.cpp:111-236.
static int restart_io(cgli_ctx *c, const char *path, int global_nx, int x_offset, bool write) {
  const int nx = c->p.nx, ny = c->p.ny, nz = c->p.nz;
  if (!path) return fail(CGLI_EINVAL, "null path");
  if (global_nx < nx || x_offset < 0 || x_offset + nx > global_nx)
    return fail(CGLI_EINVAL, "slab [x_offset, x_offset + Nx) must lie in [0, global_nx)");
  const cgli::Dev &d = c->d;
  const size_t n = (size_t)d.X * d.Y * d.Z, cells = (size_t)nx * ny * nz;
  std::vector<double> J(n), a(n), buf(cells);
  CUDA_TRY(cudaMemcpy(J.data(), d.J, n * 8, cudaMemcpyDeviceToHost));
  FILE *f = write ? fopen(path, "r+b") : fopen(path, "rb");
  if (!f && write) f = fopen(path, "w+b");
  if (!f) return fail(CGLI_EINVAL, std::string("cannot open ") + path);
  std::vector<double> U[10];
  if (!write) {
    // Initial_condition.cpp:56-103: the quiescent state on every row of the
    // interior planes, as Q/J (x ghost planes stay zero)
    const double T = 298.0592, P = 101300, rho = P / T / cgli::RG, vel = 0, VV = 0;
    const double q[5] = {rho, rho * vel, rho * vel, rho * vel, P / (cgli::KG - 1) + 0.5 * rho * VV};
    for (int f2 = 0; f2 < 10; f2++) {
      U[f2].assign(n, 0.0);
      for (int i = 3; i <= nx + 2; i++)
        for (int j = 0; j < d.Y; j++)
          for (int k = 0; k < d.Z; k++) {
            const size_t cc = cgli::ix(d, i, j, k);
            U[f2][cc] = q[f2 % 5] / J[cc];
          }
    }
  }
  int rc = CGLI_OK;
  for (int fld = 0; fld < 10 && rc == CGLI_OK; fld++) {
    const long long off = ((long long)fld * global_nx + x_offset) * (long long)ny * nz * 8;
    if (fseeko(f, (off_t)off, SEEK_SET)) { rc = fail(CGLI_EINVAL, "seek failed"); break; }
    if (write) {
      double *src = fld < 5 ? d.U[fld] : d.Uq[fld - 5];
      if (cudaMemcpy(a.data(), src, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) { rc = fail(CGLI_ECUDA, "copy"); break; }
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) {
            const size_t cc = cgli::ix(d, i + 3, j + 2, k + 2);
            buf[((size_t)i * ny + j) * nz + k] = a[cc] * J[cc];
          }
      if (fwrite(buf.data(), 8, cells, f) != cells) rc = fail(CGLI_EINVAL, std::string("short write to ") + path);
    } else {
      if (fread(buf.data(), 8, cells, f) != cells) { rc = fail(CGLI_EINVAL, std::string("short read from ") + path); break; }
      // Initial_condition.cpp:186-221
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
          for (int k = 0; k < nz; k++) {
            const size_t cc = cgli::ix(d, i + 3, j + 2, k + 2);
            U[fld][cc] = buf[((size_t)i * ny + j) * nz + k] / J[cc];
          }
    }
  }
  if (fclose(f) && rc == CGLI_OK && write) rc = fail(CGLI_EINVAL, std::string("close failed: ") + path);
  if (rc || write) return rc;
  const double *Un[5], *U0[5], *Uq[5];
  for (int v = 0; v < 5; v++) { Un[v] = U[v].data(); U0[v] = U[v].data(); Uq[v] = U[v + 5].data(); }
  return cgli_set_state(c, Un, U0, Uq);   // U_ = U (main.cpp:127-141), Q^(n-2) = Q^(n-1)
}

int cgli_write_restart(cgli_ctx *c, const char *path, int global_nx, int x_offset) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  return restart_io(c, path, global_nx, x_offset, true);
}

int cgli_read_restart(cgli_ctx *c, const char *path, int global_nx, int x_offset) {
  int rc = check(c); if (rc) return rc;
  if (!c->have_metrics) return fail(CGLI_ESTATE, "metrics not set (the reader divides by J)");
  return restart_io(c, path, global_nx, x_offset, false);
}

// sidecar of what the reference's file has no room for: the raw device
// levels U_, U, Uq, Uqq (Q/J, ghost cells included, so the lagged ghost
// values survive), the driving force, the norm maxima and the step history
struct HistoryHeader {
  char magic[8];
  int32_t nx, ny, nz, history;
  double force, emax[5];
};

int cgli_write_history(cgli_ctx *c, const char *path) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!path) return fail(CGLI_EINVAL, "null path");
  const cgli::Dev &d = c->d;
  const size_t n = (size_t)d.X * d.Y * d.Z;
  HistoryHeader h{};
  memcpy(h.magic, "CGLIHST2", 8);
  h.nx = c->p.nx; h.ny = c->p.ny; h.nz = c->p.nz; h.history = c->history; h.force = c->p.force;
  for (int v = 0; v < 5; v++) h.emax[v] = c->Emax[v];
  std::vector<double> a(n);
  FILE *f = fopen(path, "wb");
  if (!f) return fail(CGLI_EINVAL, std::string("cannot open ") + path);
  bool ok = fwrite(&h, sizeof h, 1, f) == 1;
  double *const *lv[4] = {d.U_, d.U, d.Uq, d.Uqq};
  for (int l = 0; l < 4 && ok; l++)
    for (int v = 0; v < 5 && ok; v++) {
      ok = cudaMemcpy(a.data(), lv[l][v], n * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
      if (ok) ok = fwrite(a.data(), 8, n, f) == n;
    }
  if (fclose(f)) ok = false;
  return ok ? CGLI_OK : fail(CGLI_EINVAL, std::string("write failed: ") + path);
}

int cgli_read_history(cgli_ctx *c, const char *path) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!path) return fail(CGLI_EINVAL, "null path");
  const cgli::Dev &d = c->d;
  const size_t n = (size_t)d.X * d.Y * d.Z;
  FILE *f = fopen(path, "rb");
  if (!f) return fail(CGLI_EINVAL, std::string("cannot open ") + path);
  HistoryHeader h{};
  bool ok = fread(&h, sizeof h, 1, f) == 1 && !memcmp(h.magic, "CGLIHST2", 8) && h.nx == c->p.nx &&
            h.ny == c->p.ny && h.nz == c->p.nz;
  if (!ok) { fclose(f); return fail(CGLI_EINVAL, std::string("not a history file of this grid: ") + path); }
  std::vector<double> a(n);
  double *const *lv[4] = {d.U_, d.U, d.Uq, d.Uqq};
  for (int l = 0; l < 4 && ok; l++)
    for (int v = 0; v < 5 && ok; v++) {
      ok = fread(a.data(), 8, n, f) == n;
      if (ok) ok = cudaMemcpy(lv[l][v], a.data(), n * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    }
  fclose(f);
  if (!ok) return fail(CGLI_EINVAL, std::string("short read from ") + path);
  c->history = h.history;
  for (int v = 0; v < 5; v++) c->Emax[v] = h.emax[v];
  return cgli_set_force(c, h.force);
}

int cgli_get_state(cgli_ctx *c, double *const U_[5]) {
  int rc = check(c); if (rc) return rc;
  if (!U_) return fail(CGLI_EINVAL, "null argument");
  size_t n = (size_t)c->d.X * c->d.Y * c->d.Z * sizeof(double);
  for (int v = 0; v < 5; v++) {
    if (!U_[v]) return fail(CGLI_EINVAL, "null state array");
    CUDA_TRY(cudaMemcpyAsync(U_[v], c->d.U_[v], n, cudaMemcpyDeviceToHost, c->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

#define SIMPLE_ENTRY(name, launcher, what)                  \
  int name(cgli_ctx *c) {                                   \
    int rc = check(c); if (rc) return rc;                   \
    rc = need_ready(c); if (rc) return rc;                  \
    cgli::launcher(c->d, c->stream);                        \
    rc = last_launch(what); if (rc) return rc;              \
    CUDA_TRY(cudaStreamSynchronize(c->stream));             \
    return CGLI_OK;                                         \
  }

SIMPLE_ENTRY(cgli_halo_x, launch_halo_x, "halo_x")
SIMPLE_ENTRY(cgli_y_boundary_condition, launch_bc_y, "y_boundary_condition")
SIMPLE_ENTRY(cgli_x_boundary_condition, launch_bc_x, "x_boundary_condition")
SIMPLE_ENTRY(cgli_z_boundary_condition, launch_bc_z, "z_boundary_condition")
SIMPLE_ENTRY(cgli_flux_x, launch_flux_x, "flux_x")
SIMPLE_ENTRY(cgli_flux_y, launch_flux_y, "flux_y")
SIMPLE_ENTRY(cgli_flux_z, launch_flux_z, "flux_z")
SIMPLE_ENTRY(cgli_viscous_terms, launch_viscous, "viscous_terms")

int cgli_dual_time_stepping(cgli_ctx *c, double er[5]) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!er) return fail(CGLI_EINVAL, "null er");
  cgli::launch_dts(c->d, c->stream, c->update_blocks);
  rc = last_launch("dual_time_stepping"); if (rc) return rc;
  return read_norms(c, er, c->update_blocks);
}

int cgli_dplusgs(cgli_ctx *c, double er[5]) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!er) return fail(CGLI_EINVAL, "null er");
  if (c->p.precision != CGLI_FP64) return fail(CGLI_EINVAL, "DP-LUR needs precision CGLI_FP64");
  cgli::launch_dplur(c->d, c->sw, c->stream);
  rc = last_launch("dplusgs"); if (rc) return rc;
  return read_norms(c, er, c->update_blocks);
}

int cgli_set_inner_solver(cgli_ctx *c, int solver) {
  int rc = check(c); if (rc) return rc;
  if (solver != CGLI_LUSGS && solver != CGLI_DPLUR)
    return fail(CGLI_EINVAL, "inner solver must be CGLI_LUSGS or CGLI_DPLUR");
  if (solver == CGLI_DPLUR && c->p.precision != CGLI_FP64)
    return fail(CGLI_EINVAL, "DP-LUR needs precision CGLI_FP64");
  if (solver != c->inner_solver) drop_graph(c);
  c->inner_solver = solver;
  return CGLI_OK;
}

int cgli_inner_iteration(cgli_ctx *c, double er[5]) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!er) return fail(CGLI_EINVAL, "null er");
  if (!c->metrics_checked) {
    rc = check_channel_metrics(c); if (rc) return rc;
  }
  const bool dplur = c->inner_solver == CGLI_DPLUR;
  if (!c->iter_graph) {
    cudaGraph_t g;
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    if (dplur) {
      cgli::launch_dplur_iteration(c->d, c->sw, c->stream);
    } else {
      // the four wavefront passes are bracketed by two events, so that their
      // device time is known for every iteration the graph runs
      cgli::launch_fused_residual(c->d, c->sw, c->stream, c->p.precision);
      // (external records: event-record nodes of the graph, not capture-internal dependencies)
      cudaEventRecordWithFlags(c->sweep_ev[0], c->stream, cudaEventRecordExternal);
      cgli::launch_sweeps(c->d, c->sw, c->stream, c->p.precision == CGLI_MIXED);
      cudaEventRecordWithFlags(c->sweep_ev[1], c->stream, cudaEventRecordExternal);
      cgli::launch_sweep_update(c->d, c->sw, c->stream, c->p.precision == CGLI_MIXED);
    }
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->iter_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  CUDA_TRY(cudaGraphLaunch(c->iter_graph, c->stream));
  rc = read_norms(c, er, dplur ? c->update_blocks : c->sweep_update_blocks);   // synchronises the stream
  if (rc == CGLI_OK && !dplur) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, c->sweep_ev[0], c->sweep_ev[1]) == cudaSuccess) {
      c->sweep_ms += ms;
      c->sweep_passes += 4;
    } else {
      cudaGetLastError();   // timing unavailable: leave no error behind for the next call
    }
  }
  return rc;
}

int cgli_driven_force(cgli_ctx *c, double *bulk_flux) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!bulk_flux) return fail(CGLI_EINVAL, "null argument");
  cgli::launch_bulk_flux(c->d, c->stream, c->d_out);
  rc = last_launch("driven_force"); if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(c->h_norms, c->d_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  *bulk_flux = c->h_norms[0];
  return CGLI_OK;
}

int cgli_end_step(cgli_ctx *c) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  cgli::launch_end_step(c->d, c->stream);
  rc = last_launch("end_step"); if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

int cgli_set_force(cgli_ctx *c, double force) {
  int rc = check(c); if (rc) return rc;
  c->p.force = force;
  CUDA_TRY(cudaMemcpyAsync(c->d.scal, &c->p.force, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

int cgli_set_predictor(cgli_ctx *c, int mode) {
  int rc = check(c); if (rc) return rc;
  if (mode < 0 || mode > 2)
    return fail(CGLI_EINVAL, "predictor mode must be 0 (previous level), 1 (extrapolation) or 2 (learned)");
  if (mode == 2 && !c->cnn) return fail(CGLI_ESTATE, "predictor 2 needs a network (cgli_set_learned_guess)");
  c->predictor = mode;
  return CGLI_OK;
}

int cgli_sweep_tile_shape(int precision, int *ti, int *tj) {
  if (!ti || !tj) return fail(CGLI_EINVAL, "null argument");
  if (precision != CGLI_FP64 && precision != CGLI_MIXED)
    return fail(CGLI_EINVAL, "precision must be CGLI_FP64 or CGLI_MIXED");
  *ti = precision == CGLI_MIXED ? cgli::SweepTile<float>::TI : cgli::SweepTile<double>::TI;
  *tj = precision == CGLI_MIXED ? cgli::SweepTile<float>::TJ : cgli::SweepTile<double>::TJ;
  return CGLI_OK;
}

int cgli_set_wait_limit(cgli_ctx *c, int polls) {
  int rc = check(c); if (rc) return rc;
  if (polls < 0) return fail(CGLI_EINVAL, "wait limit must be >= 0 polls");
  if (polls != c->sw.spin_limit) drop_graph(c);   // the graph holds the launch arguments
  c->sw.spin_limit = polls;
  return CGLI_OK;
}

int cgli_filter(cgli_ctx *c, double roe_criterion, double e_high, double e_low) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!c->have_ypoint) return fail(CGLI_ESTATE, "Y_point not set (cgli_set_array(ctx, \"Y_point\", ...))");
  rc = ensure_filter(c); if (rc) return rc;
  CUDA_TRY(cgli::launch_filter(c->d, c->fb, roe_criterion, e_high, e_low, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CGLI_OK;
}

int cgli_step_norms(cgli_ctx *c, double *norms, int max_iters, int *iters) {
  int rc = check(c); if (rc) return rc;
  if (!norms || !iters || max_iters < 0) return fail(CGLI_EINVAL, "null argument");
  const int n = (int)(c->step_norms.size() / 5);
  *iters = n;
  std::copy(c->step_norms.begin(), c->step_norms.begin() + 5 * std::min(n, max_iters), norms);
  return CGLI_OK;
}

int cgli_statistics_accumulate(cgli_ctx *c) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  const size_t bytes = (size_t)CGLI_NSTATS * c->p.nx * c->p.ny * sizeof(double);
  if (!c->stats) { rc = alloc(c, bytes, (void **)&c->stats); if (rc) return rc; }
  cgli::launch_statistics(c->d, c->stream, c->stats);
  rc = last_launch("statistics"); if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->stat_samples++;
  return CGLI_OK;
}

int cgli_statistics_get(cgli_ctx *c, double *sums, long long *samples) {
  int rc = check(c); if (rc) return rc;
  if (!sums || !samples) return fail(CGLI_EINVAL, "null argument");
  const size_t bytes = (size_t)CGLI_NSTATS * c->p.nx * c->p.ny * sizeof(double);
  if (!c->stats) memset(sums, 0, bytes);
  else {
    CUDA_TRY(cudaMemcpyAsync(sums, c->stats, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  *samples = c->stat_samples;
  return CGLI_OK;
}

int cgli_statistics_reset(cgli_ctx *c) {
  int rc = check(c); if (rc) return rc;
  if (c->stats) {
    CUDA_TRY(cudaMemsetAsync(c->stats, 0, (size_t)CGLI_NSTATS * c->p.nx * c->p.ny * sizeof(double), c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  c->stat_samples = 0;
  return CGLI_OK;
}

int cgli_set_learned_guess(cgli_ctx *c, cgli_cnn *n) {
  int rc = check(c); if (rc) return rc;
  if (n && !cgli::cnn_matches(n, c->p.nx, c->p.ny, c->p.nz))
    return fail(CGLI_EINVAL, "network grid differs from the context's grid");
  c->cnn = n;
  if (!n && c->predictor == 2) c->predictor = 1;
  return CGLI_OK;
}

int cgli_cnn_push_level(cgli_cnn *n, cgli_ctx *c) {
  int rc = check(c); if (rc) return rc;
  if (!n || !cgli::cnn_matches(n, c->p.nx, c->p.ny, c->p.nz))
    return fail(CGLI_EINVAL, "network grid differs from the context's grid");
  if (!c->have_state) return fail(CGLI_ESTATE, "state not set (cgli_set_state)");
  return cgli::cnn_store_level(n, c->d, c->stream);
}

int cgli_cnn_time_inference(cgli_cnn *n, cgli_ctx *c, int reps, float *ms) {
  int rc = check(c); if (rc) return rc;
  if (!n || !ms || reps <= 0) return fail(CGLI_EINVAL, "bad argument");
  if (!cgli::cnn_matches(n, c->p.nx, c->p.ny, c->p.nz)) return fail(CGLI_EINVAL, "network grid differs from the context's grid");
  if (!c->have_state) return fail(CGLI_ESTATE, "state not set (cgli_set_state)");
  return cgli::cnn_time_inference(n, c->d, c->stream, reps, ms);
}

int cgli_step(cgli_ctx *c, int fixed_iters, double drop, int cap, int *iters, double er[5]) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!iters || !er) return fail(CGLI_EINVAL, "null argument");
  if (fixed_iters <= 0 && (cap <= 0 || !(drop > 0))) return fail(CGLI_EINVAL, "need fixed_iters > 0 or cap > 0 and drop > 0");
  if (c->predictor == 2 && c->history >= 2) {
    CUDA_TRY(cgli::cnn_predict(c->cnn, c->d, c->stream));
  } else if (c->predictor >= 1 && c->history >= 1) {
    // extrapolation, also the learned guess's fallback without two levels of history
    cgli::launch_predict(c->d, c->stream, c->history >= 2 ? 2 : 1);
    rc = last_launch("predict"); if (rc) return rc;
  }
  int it = 0;
  c->step_norms.clear();
  while (true) {
    it++;
    rc = cgli_inner_iteration(c, er);
    if (rc) return rc;
    c->step_norms.insert(c->step_norms.end(), er, er + 5);
    // main.cpp:287-304: norms divided by their running maximum over the run
    bool done = true;
    for (int v = 0; v < 5; v++) {
      c->Emax[v] = std::max(c->Emax[v], er[v]);
      done = done && (c->Emax[v] > 0 ? er[v] / c->Emax[v] < drop : true);
    }
    if (fixed_iters > 0) {
      if (it >= fixed_iters) break;
    } else if (done || it >= cap) {
      break;
    }
  }
  *iters = it;
  rc = cgli_end_step(c);
  if (rc == CGLI_OK) c->history++;
  return rc;
}

static int copy_metric(const cgli::MetricSet &M, const char *name, double *out);

int cgli_channel_metrics_host(int nx, int ny, int nz, double det, double high, double stretch,
                              const char *name, double *out) {
  if (!name || !out || nx < 1 || ny < 1 || nz < 1 || !(det > 0 && high > 0 && stretch > 0))
    return fail(CGLI_EINVAL, "bad argument");
  cgli::MetricSet M;
  cgli::channel_metrics(nx, ny, nz, det, high, stretch, M);
  return copy_metric(M, name, out);
}

int cgli_wavy_channel_metrics_host(int nx, int ny, int nz, double dxi, double det, double high, double stretch,
                                   double amplitude, const char *name, double *out) {
  if (!name || !out || nx < 1 || ny < 1 || nz < 1 || !(dxi > 0 && det > 0 && high > 0 && stretch > 0) ||
      !(fabs(amplitude) < 0.5 * high))
    return fail(CGLI_EINVAL, "bad argument");
  cgli::MetricSet M;
  cgli::wavy_metrics(nx, ny, nz, dxi, det, high, stretch, amplitude, M);
  return copy_metric(M, name, out);
}

static int copy_metric(const cgli::MetricSet &M, const char *name, double *out) {
  const std::vector<double> *src = nullptr;
  if (!strcmp(name, "J")) src = &M.J;
  const char *fs[3] = {"J_u", "J_v", "J_w"};
  const char *sfx[3] = {"_u", "_v", "_w"};
  char buf[32];
  for (int f = 0; f < 3 && !src; f++)
    if (!strcmp(name, fs[f])) src = &M.Jf[f];
  for (int v = 0; v < 9 && !src; v++) {
    if (!strcmp(name, kMetricNames[v])) src = &M.m[v];
    for (int f = 0; f < 3 && !src; f++) {
      snprintf(buf, sizeof buf, "%s%s", kMetricNames[v], sfx[f]);
      if (!strcmp(name, buf)) src = &M.mf[f][v];
    }
  }
  if (!src) return fail(CGLI_EINVAL, std::string("unknown metric ") + name);
  memcpy(out, src->data(), src->size() * sizeof(double));
  return CGLI_OK;
}

int cgli_event_record(cgli_ctx *c, int slot) {
  int rc = check(c); if (rc) return rc;
  if (slot < 0 || slot >= 8) return fail(CGLI_EINVAL, "event slot out of range");
  CUDA_TRY(cudaEventRecord(c->events[slot], c->stream));
  return CGLI_OK;
}

int cgli_sweep_time(cgli_ctx *c, double *ms, long long *passes, int reset) {
  int rc = check(c); if (rc) return rc;
  if (!ms || !passes) return fail(CGLI_EINVAL, "null argument");
  *ms = c->sweep_ms;
  *passes = c->sweep_passes;
  if (reset) { c->sweep_ms = 0; c->sweep_passes = 0; }
  return CGLI_OK;
}

int cgli_event_elapsed(cgli_ctx *c, int a, int b, float *ms) {
  int rc = check(c); if (rc) return rc;
  if (a < 0 || a >= 8 || b < 0 || b >= 8 || !ms) return fail(CGLI_EINVAL, "bad argument");
  CUDA_TRY(cudaEventSynchronize(c->events[b]));
  CUDA_TRY(cudaEventElapsedTime(ms, c->events[a], c->events[b]));
  return CGLI_OK;
}

int cgli_profile_stages(cgli_ctx *c, int reps, double *ms) {
  int rc = check(c); if (rc) return rc;
  rc = need_ready(c); if (rc) return rc;
  if (!ms || reps < 1) return fail(CGLI_EINVAL, "bad argument");
  if (!c->metrics_checked) { rc = check_channel_metrics(c); if (rc) return rc; }
  const bool mixed = c->p.precision == CGLI_MIXED;
  cudaEvent_t ev[CGLI_NSTAGES + 1];
  for (auto &e : ev) CUDA_TRY(cudaEventCreate(&e));
  double tot[CGLI_NSTAGES] = {0};
  for (int r = 0; r < reps; r++) {
    // the sweep stages stand for two passes each; time the first of each kind
    CUDA_TRY(cudaEventRecord(ev[0], c->stream));
    cgli::launch_halo_bc(c->d, c->stream);
    CUDA_TRY(cudaEventRecord(ev[1], c->stream));
    cgli::launch_flux_x(c->d, c->stream);
    CUDA_TRY(cudaEventRecord(ev[2], c->stream));
    cgli::launch_flux_y(c->d, c->stream);
    CUDA_TRY(cudaEventRecord(ev[3], c->stream));
    cgli::launch_flux_z(c->d, c->stream);
    CUDA_TRY(cudaEventRecord(ev[4], c->stream));
    cgli::launch_viscous(c->d, c->stream);
    CUDA_TRY(cudaEventRecord(ev[5], c->stream));
    cgli::launch_residual_fast(c->d, c->sw, c->stream, mixed);
    CUDA_TRY(cudaEventRecord(ev[6], c->stream));
    cgli::launch_sweep_pass(c->d, c->sw, c->stream, mixed, false, false);
    CUDA_TRY(cudaEventRecord(ev[7], c->stream));
    cgli::launch_sweep_pass(c->d, c->sw, c->stream, mixed, true, false);
    CUDA_TRY(cudaEventRecord(ev[8], c->stream));
    cgli::launch_sweep_pass(c->d, c->sw, c->stream, mixed, false, false);
    cgli::launch_sweep_pass(c->d, c->sw, c->stream, mixed, true, true);
    rc = last_launch("profile_stages"); if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < CGLI_NSTAGES; s++) {
      float t = 0;
      CUDA_TRY(cudaEventElapsedTime(&t, ev[s], ev[s + 1]));
      tot[s] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  for (int s = 0; s < CGLI_NSTAGES; s++) ms[s] = tot[s] / reps;
  return CGLI_OK;
}

int cgli_hyperplane(int nx, int ny, int nz, int *Nijk, long nijk_len, int *ijk, long ijk_len) {
  if (!Nijk || !ijk || nx < 1 || ny < 1 || nz < 1) return fail(CGLI_EINVAL, "bad argument");
  if (!cgli::hyperplane(nx, ny, nz, Nijk, nijk_len, ijk, ijk_len)) return fail(CGLI_EINVAL, "buffers too small");
  return CGLI_OK;
}

}  // extern "C"
