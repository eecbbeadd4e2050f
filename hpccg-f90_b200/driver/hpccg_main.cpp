// hpccg_main.cpp -- host driver mirroring MPI/src/main.F90 (HPCCGmain, printInfo).
//
// The reference keeps its driver in Fortran 90; without a Fortran compiler at
// hand, this C++ program is the host side above the
// C-ABI: same command line (`nx ny nz`), same generate_matrix -> printInfo ->
// cg(max_iter=150, tolerance=0) sequence (main.F90:103-130), same report lines
// (numerics.F90:103,125,150).  Extra options keep the reference defaults.
//
//   HPCCG-B200 nx ny nz [--max-iter N] [--tol T] [--device-generate]
//                       [--spmv KIND[,PARAM]] [--timing-level L] [--quiet]
//
// --timing-level follows the reference's TIMINGLEV (MPI/config.mk TIMER_LEVEL,
// default 1; numerics.F90:100-156): 1 prints "TIMER: Total"; 2 adds one
// "TIMER: Iteration" line per iteration; 3 adds "MFLOPS SPARSEMV" with the
// reference's operation count niters * 2 * total_nnz (total_nnz = 27 N).  The
// whole CG runs as one graph launch, so the per-iteration figure is the device
// solve time divided by the iteration count, and the SpMV time is the fused
// SpMV kernel's measured time per launch times the iteration count.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hpccg_gpu.h"

// Fortran `e20.10` edit descriptor: 0.dddddddddd E+xx, right-aligned in 20.
static std::string fortran_e(double v, int w = 20, int d = 10) {
  char buf[64];
  if (!std::isfinite(v)) {
    snprintf(buf, sizeof buf, "%*s", w, std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
    return buf;
  }
  int e = 0;
  double m = std::fabs(v);
  if (m != 0.0) {
    // scientific with d digits gives 1 <= |mant| < 10; shift to 0.1 <= mant < 1
    char tmp[64];
    snprintf(tmp, sizeof tmp, "%.*e", d - 1, m);
    const char *ep = strchr(tmp, 'e');
    e = atoi(ep + 1) + 1;
    std::string digits;
    for (const char *q = tmp; q < ep; ++q)
      if (*q >= '0' && *q <= '9') digits.push_back(*q);
    snprintf(buf, sizeof buf, "%s0.%sE%c%02d", v < 0 ? "-" : "", digits.c_str(), e < 0 ? '-' : '+',
             std::abs(e));
  } else {
    snprintf(buf, sizeof buf, "0.%sE+00", std::string(d, '0').c_str());
  }
  char out[64];
  snprintf(out, sizeof out, "%*s", w, buf);
  return out;
}

static void check(int rc, const char *what) {
  if (rc != HPCCG_OK) {
    fprintf(stderr, "HPCCG-B200: %s: %s\n", what, hpccg_strerror(rc));
    exit(1);
  }
}

int main(int argc, char **argv) {
  if (argc < 4) {
    printf(" USAGE: ./HPCCG <nx> <ny> <nz>\n");
    return 0;
  }
  const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
  int max_iter = 150;    // main.F90:127
  double tolerance = 0;  // main.F90:128
  bool device_generate = false, quiet = false;
  int timing_level = 1;  // MPI/config.mk TIMER_LEVEL
  int spmv_kind = HPCCG_SPMV_AUTO, spmv_param = 0;
  for (int i = 4; i < argc; ++i) {
    if (!strcmp(argv[i], "--max-iter") && i + 1 < argc) max_iter = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--tol") && i + 1 < argc) tolerance = atof(argv[++i]);
    else if (!strcmp(argv[i], "--device-generate")) device_generate = true;
    else if (!strcmp(argv[i], "--quiet")) quiet = true;
    else if (!strcmp(argv[i], "--timing-level") && i + 1 < argc) timing_level = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--spmv") && i + 1 < argc) {
      spmv_kind = atoi(argv[++i]);
      const char *comma = strchr(argv[i], ',');
      if (comma) spmv_param = atoi(comma + 1);
    } else {
      fprintf(stderr, "HPCCG-B200: unknown option %s\n", argv[i]);
      return 2;
    }
  }
  if (nx < 1 || ny < 1 || nz < 1) {
    fprintf(stderr, "HPCCG-B200: nx, ny, nz must be positive\n");
    return 2;
  }
  const int64_t n = (int64_t)nx * ny * nz;
  std::vector<double> x(n), b(n), xexact(n);
  hpccg_ctx *ctx = nullptr;
  int64_t nnz = 0;
  if (device_generate) {
    // A is built on the device; x0, b and xexact follow from the row's kept
    // neighbour count, b = 27 - (nnzrow - 1) (SparseMatrix.F90:170-172).
    check(hpccg_gpu_create_generated(nx, ny, nz, nullptr, nullptr, nullptr, &ctx), "generate");
    check(hpccg_gpu_info(ctx, nullptr, &nnz, nullptr), "info");
    auto kept = [](int i, int m) { return 1 + (i > 1) + (i < m); };
    for (int64_t r = 0; r < n; ++r) {
      const int ix = (int)(r % nx) + 1, iy = (int)((r / nx) % ny) + 1, iz = (int)(r / ((int64_t)nx * ny)) + 1;
      x[r] = 0.0;
      b[r] = 27.0 - (double)(kept(ix, nx) * kept(iy, ny) * kept(iz, nz) - 1);
      xexact[r] = 1.0;
    }
  } else {
    std::vector<int32_t> rowindex(n + 1), colindex(27 * n);
    std::vector<double> values(27 * n);
    check(hpccg_generate_matrix(nx, ny, nz, rowindex.data(), colindex.data(), values.data(), x.data(),
                                b.data(), xexact.data(), &nnz),
          "generate_matrix");
    check(hpccg_gpu_create((int32_t)n, nnz, rowindex.data(), colindex.data(), values.data(), &ctx),
          "create");
  }
  if (spmv_kind == HPCCG_SPMV_STENCIL && !device_generate)
    check(hpccg_gpu_set_geometry(ctx, nx, ny, nz), "set_geometry");  // device check of the CSR
  if (spmv_kind != HPCCG_SPMV_AUTO) check(hpccg_gpu_set_spmv(ctx, spmv_kind, spmv_param), "set_spmv");

  // printInfo, main.F90:33-75 (total_nnz is the reference's 27*N count)
  printf(" HPCCG Benchmark\n");
  printf(" Using double precision\n");
  printf(" Total size (N x N): %12lld\n", (long long)n);
  printf(" Total nonzeroes: %12lld\n", (long long)(27 * n));
  printf(" MPI disabled.\n");
  printf(" OpenMP disabled.\n");
  printf(" GPU: sm_100a kernels, stored nonzeroes %lld\n", (long long)nnz);

  std::vector<double> hist(max_iter + 1);
  int32_t niters = 0;
  double normr = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = hpccg_gpu_cg(ctx, b.data(), x.data(), max_iter, tolerance, &niters, &normr, hist.data());
  const auto t1 = std::chrono::steady_clock::now();
  if (rc != HPCCG_OK && rc != HPCCG_ERR_BREAKDOWN) check(rc, "cg");

  // numerics.F90:103 and :123-126 (print_freq = clamp(max_iter/10, 1, 50))
  printf(" Initial Residual = %25.17g\n", hist[0]);
  if (!quiet) {
    int print_freq = max_iter / 10;
    if (print_freq > 50) print_freq = 50;
    if (print_freq < 1) print_freq = 1;
    for (int k = 1; k <= niters; ++k)
      if (k % print_freq == 0 || k + 1 == max_iter)
        printf("ITER%5d  Residual%s\n", k, fortran_e(hist[k]).c_str());
  }
  if (rc == HPCCG_ERR_BREAKDOWN) printf(" CG breakdown after %d iterations\n", niters);
  const double secs = std::chrono::duration<double>(t1 - t0).count();
  float solve_ms = 0.f;
  check(hpccg_gpu_last_solve_ms(ctx, &solve_ms), "last_solve_ms");
  if (timing_level > 1 && niters > 0)
    for (int k = 1; k <= niters; ++k) printf(" TIMER: Iteration %15.7g sec\n", 1e-3 * solve_ms / niters);
  if (timing_level > 0) printf(" TIMER: Total %15.7g sec\n", secs);
  if (timing_level > 2 && niters > 0) {
    float kms[3] = {0.f, 0.f, 0.f};
    check(hpccg_gpu_time_cg_kernels(ctx, 10, kms), "time_cg_kernels");
    const double total_time_spmv = 1e-3 * kms[1] * niters;
    const double fnops_sparsemv = niters * 2.0 * (double)(27 * n);
    printf(" MFLOPS SPARSEMV %15.7g\n", fnops_sparsemv / total_time_spmv / 1.0e6);
  }
  double err = 0.0;
  for (int64_t i = 0; i < n; ++i) err = std::fmax(err, std::fabs(x[i] - xexact[i]));
  printf(" Iterations: %d  final normr: %.17g  max|x - xexact|: %.3e\n", niters, normr, err);
  hpccg_gpu_destroy(ctx);
  return rc == HPCCG_OK ? 0 : 3;
}
