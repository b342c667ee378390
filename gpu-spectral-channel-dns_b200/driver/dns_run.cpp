// The parameter.txt driver (the reference's run_simulation,
// source/main_loop.cpp:15-115) over libdnsb200's C ABI.
//
//   dns_run [parameter.txt] [--mixed] [--device N] [--recovery FILE] [--print-every K]
//
// start_type 0: the analytic start (initFlow), its fields written as step 0,
// the nonlinear history of the initial state (the reference's "extra
// previous step"), then one step (the reference's "first step"); start_type
// 1: state and history from the recovery file (the reference's fixed name
// recovery.dat unless --recovery is given).  Then steps start_step ..
// end_step; fields every save_internal steps, the recovery file every
// save_recovery_internal steps (not at step 0).  Each step prints its time
// and the mean; v-hat of mode (0,0), wall-normal coefficient 0, is printed at
// output steps and every --print-every steps (reading it copies the state to
// the host).  A state that turns NaN or Inf ends the run (exit status 3).
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dns_b200.h"

static void check(dns_status s, const char* what) {
  if (s != DNS_OK) {
    std::fprintf(stderr, "dns_run: %s: %s (%s)\n", what, dns_status_string(s), dns_last_error());
    std::exit(2);
  }
}

int main(int argc, char** argv) {
  std::string param = "../input/parameter.txt", recovery = "recovery.dat";
  int device = 0, precision = DNS_PREC_FP64, print_every = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--mixed") precision = DNS_PREC_MIXED;
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (a == "--recovery" && i + 1 < argc) recovery = argv[++i];
    else if (a == "--print-every" && i + 1 < argc) print_every = std::atoi(argv[++i]);
    else if (a == "-h" || a == "--help") {
      std::printf("usage: dns_run [parameter.txt] [--mixed] [--device N] [--recovery FILE] [--print-every K]\n");
      return 0;
    } else if (!a.empty() && a[0] == '-') {
      std::fprintf(stderr, "dns_run: unknown option %s\n", a.c_str());
      return 1;
    } else {
      param = a;
    }
  }
  std::printf("Reading settings from %s\n", param.c_str());
  dns_params p;
  dns_run_params rp;
  check(dns_read_parameter_file(param.c_str(), &p, &rp), "parameter file");
  if (rp.save_internal <= 0 || rp.save_recovery_internal <= 0) {
    std::fprintf(stderr, "dns_run: save intervals must be positive\n");
    return 1;
  }
  p.precision = precision;
  p.device = device;
  dns_ctx* ctx = nullptr;
  check(dns_create(&p, &ctx), "create");
  int geo[8];
  check(dns_geometry(ctx, geo), "geometry");
  const int Ny = geo[1], Nz = geo[2], Kx = geo[3];
  std::vector<std::complex<double>> v((size_t)Nz * Kx * Ny), om(v.size());
  const std::string pre = rp.output_file_prefix;
  auto write_fields = [&](int step) {
    const std::string s = std::to_string(step);
    check(dns_write_fields(ctx, (pre + "_velocity." + s + ".dat").c_str(),
                           (pre + "_vortricity." + s + ".dat").c_str()),
          "field output");
  };
  if (rp.start_type == 0) {
    std::printf("init flow\n");
    check(dns_init_flow(ctx), "initFlow");
    std::printf("output initial flow field\n");
    write_fields(0);
    std::printf("extra previous step\n");
    check(dns_bootstrap(ctx), "bootstrap");
    std::printf("first step\n");
    check(dns_step(ctx, 1), "step");
  } else if (rp.start_type == 1) {
    check(dns_read_recovery(ctx, recovery.c_str()), "recovery file");
  } else {
    std::fprintf(stderr, "wrong start type\n");
    dns_destroy(ctx);
    return 1;
  }
  double total = 0.0;
  int count = 0;
  for (int i = rp.start_step; i <= rp.end_step; ++i) {
    std::printf("\nSTEP: %d\n", i);
    const auto t0 = std::chrono::steady_clock::now();
    check(dns_step(ctx, 1), "step");
    check(dns_synchronize(ctx), "step");
    const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const dns_status cs = dns_check_state(ctx);
    if (cs == DNS_ERR_NONFINITE) {
      std::fprintf(stderr, "dns_run: the state holds NaN or Inf after step %d\n", i);
      dns_destroy(ctx);
      return 3;
    }
    check(cs, "state check");  // any other failure of the check ends the run (status 2)
    total += t;
    ++count;
    std::printf("Time cost of current step:%g\nMean time cost per step:%g\n", t, total / count);
    const bool out = i % rp.save_internal == 0;
    if (out || (print_every > 0 && i % print_every == 0)) {
      check(dns_get_state(ctx, v.data(), om.data(), (size_t)Ny * 16, DNS_HOST), "state");
      std::printf("velocity(0,0,0):%.17g %.17g\n", v[0].real(), v[0].imag());
    }
    if (out) {
      std::printf("[OUTPUT] WRITING RESULTS\n");
      write_fields(i);
    }
    if (i % rp.save_recovery_internal == 0 && i > 0) {
      std::printf("[OUTPUT] WRITING RECOVERY FILES\n");
      check(dns_write_recovery(ctx, recovery.c_str()), "recovery file");
    }
  }
  check(dns_destroy(ctx), "destroy");
  return 0;
}
