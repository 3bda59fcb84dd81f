// Host driver in the reference's own language: the physical-step loop of
// main.cpp:143-404 on top of the C ABI of include/cgli_fu_flow.h.
//
// Reads the initial field from a restart file in the reference's layout
// (Initial_condition.cpp with switch_initial = 1), runs K physical steps
// (inner iterations until the stopping rule of main.cpp:287-304, or a fixed
// count), updates the driving force once per step from the bulk flux
// (Driven_force.cpp:14-74 plus the mass-flux controller of the workloads, or
// a fixed force), prints one line per step as main.cpp:313 does, and writes
// the final state in the LES%05d.bin layout of Output.cpp:187-284.
//
//   cgli_run --nx N --ny N --nz N --dxi D --det D --dzt D --dt D --e E --mu M --pr P
//            --high H --stretch G --initial FILE --steps K [--output FILE]
//            [--fixed ITERS | --drop 1e-3 --cap 30] [--twall-lo T --twall-hi T]
//            [--mixed] [--dplur] [--predictor 0|1] [--open NIN NOUT] [--buoyancy]
//            [--force F | --target-flux Q --force-lam F0 [--kp 0.5] [--ki 0.05]]
//
// Exit status: 0 on success, 1 on a bad command line, 2 on a library error
// (its message on stderr).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cgli_fu_flow.h"

namespace {

void usage(FILE *f) {
  std::fprintf(f,
               "usage: cgli_run --nx N --ny N --nz N --dxi D --det D --dzt D --dt D --e E --mu M --pr P\n"
               "                --high H --stretch G --initial FILE --steps K [--output FILE]\n"
               "                [--fixed ITERS | --drop D --cap C] [--twall-lo T --twall-hi T]\n"
               "                [--mixed] [--dplur] [--predictor 0|1] [--open NIN NOUT] [--buoyancy]\n"
               "                [--force F | --target-flux Q --force-lam F0 [--kp KP] [--ki KI]]\n");
}

int fail(const char *what) {
  std::fprintf(stderr, "cgli_run: %s: %s\n", what, cgli_last_error());
  return 2;
}

}  // namespace

int main(int argc, char **argv) {
  cgli_params p;
  std::memset(&p, 0, sizeof p);
  p.twall_lo = p.twall_hi = 298.0592;   // Y_boundary_condition.cpp:166
  p.precision = CGLI_FP64;
  double stretch = 0, force = 0, target = 0, force_lam = 0, kp = 0.5, ki = 0.05, drop = 1e-3;
  int steps = 0, fixed = 0, cap = 30, predictor = 0, dplur = 0, controlled = 0;
  const char *initial = nullptr, *output = nullptr;
  for (int a = 1; a < argc; a++) {
    const std::string o = argv[a];
    auto val = [&](int k = 1) -> const char * {
      if (a + k >= argc) { usage(stderr); std::exit(1); }
      return argv[a + k];
    };
    if (o == "--help" || o == "-h") { usage(stdout); return 0; }
    else if (o == "--nx") p.nx = std::atoi(val()), a++;
    else if (o == "--ny") p.ny = std::atoi(val()), a++;
    else if (o == "--nz") p.nz = std::atoi(val()), a++;
    else if (o == "--dxi") p.dxi = std::atof(val()), a++;
    else if (o == "--det") p.det = std::atof(val()), a++;
    else if (o == "--dzt") p.dzt = std::atof(val()), a++;
    else if (o == "--dt") p.dt = std::atof(val()), a++;
    else if (o == "--e") p.e = std::atof(val()), a++;
    else if (o == "--mu") p.mu = std::atof(val()), a++;
    else if (o == "--pr") p.pr = std::atof(val()), a++;
    else if (o == "--high") p.high = std::atof(val()), a++;
    else if (o == "--stretch") stretch = std::atof(val()), a++;
    else if (o == "--twall-lo") p.twall_lo = std::atof(val()), a++;
    else if (o == "--twall-hi") p.twall_hi = std::atof(val()), a++;
    else if (o == "--initial") initial = val(), a++;
    else if (o == "--output") output = val(), a++;
    else if (o == "--steps") steps = std::atoi(val()), a++;
    else if (o == "--fixed") fixed = std::atoi(val()), a++;
    else if (o == "--drop") drop = std::atof(val()), a++;
    else if (o == "--cap") cap = std::atoi(val()), a++;
    else if (o == "--predictor") predictor = std::atoi(val()), a++;
    else if (o == "--mixed") p.precision = CGLI_MIXED;
    else if (o == "--dplur") dplur = 1;
    else if (o == "--buoyancy") p.buoyancy = 1;
    else if (o == "--open") { p.x_open = 1; p.nx_inlet = std::atoi(val(1)); p.nx_outlet = std::atoi(val(2)); a += 2; }
    else if (o == "--force") force = std::atof(val()), a++;
    else if (o == "--target-flux") target = std::atof(val()), controlled = 1, a++;
    else if (o == "--force-lam") force_lam = std::atof(val()), a++;
    else if (o == "--kp") kp = std::atof(val()), a++;
    else if (o == "--ki") ki = std::atof(val()), a++;
    else { std::fprintf(stderr, "cgli_run: unknown option %s\n", o.c_str()); usage(stderr); return 1; }
  }
  if (!initial || steps <= 0 || p.nx <= 0 || !(stretch > 0) || !(p.high > 0)) { usage(stderr); return 1; }
  if (controlled) force = force_lam;
  p.force = force;

  cgli_ctx *ctx = nullptr;
  if (cgli_create(&p, &ctx)) return fail("cgli_create");
  int rc = 0;
  double integral = 0;   // controller state
  // main.cpp:87-141: metrics (Jacobian*.cpp), then the initial field
  if (cgli_channel_metrics(ctx, p.high, stretch)) { rc = fail("cgli_channel_metrics"); goto done; }
  if (cgli_read_restart(ctx, initial, p.nx, 0)) { rc = fail("cgli_read_restart"); goto done; }
  if (cgli_set_force(ctx, force)) { rc = fail("cgli_set_force"); goto done; }
  if (dplur && cgli_set_inner_solver(ctx, CGLI_DPLUR)) { rc = fail("cgli_set_inner_solver"); goto done; }
  if (predictor && cgli_set_predictor(ctx, predictor)) { rc = fail("cgli_set_predictor"); goto done; }
  for (int step = 1; step <= steps; step++) {
    int it = 0;
    double er[5];
    if (cgli_step(ctx, fixed, drop, cap, &it, er)) { rc = fail("cgli_step"); goto done; }
    if (controlled) {
      // bulk flux of the converged level and the workloads' mass-flux
      // controller: e = Q_target - Q_b, I += e, F = F_lam + (kp e + ki I)/dt
      double qb = 0;
      if (cgli_driven_force(ctx, &qb)) { rc = fail("cgli_driven_force"); goto done; }
      const double e = target - qb;
      integral = integral + e;
      force = force_lam + (kp * e + ki * integral) / p.dt;
      if (cgli_set_force(ctx, force)) { rc = fail("cgli_set_force"); goto done; }
    }
    std::printf("%d\t%d\t%.9e\t%.9e\t%.9e\t%.9e\t%.9e\t%.17g\n", step, it, er[0], er[1], er[2], er[3], er[4], force);
    std::fflush(stdout);
  }
  if (output && cgli_write_restart(ctx, output, p.nx, 0)) rc = fail("cgli_write_restart");
done:
  cgli_destroy(ctx);
  return rc;
}
