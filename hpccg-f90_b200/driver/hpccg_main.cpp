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
//                       [--precision fp64|fp32|bf16] [--rel-tol R]
//   HPCCG-B200 --batch SPEC [--precision ...] [--rel-tol R] [--max-iter N] [--spmv 4]
//   HPCCG-B200 nx ny nz --ranks P [--halo mpi|get] [--max-iter N] [--tol T] [--quiet]
//
// --precision fp32 or bf16 replaces the reference's fixed-count CG by the
// FP64 iterative refinement around a low-precision inner CG
// (hpccg_gpu_solve_mixed), run to the FP64 relative residual --rel-tol
// (default 1e-8); fp64 (the default) is the reference's CG.  --batch solves
// many generate_matrix systems of the reference's problem (x0 = 0, b = A 1)
// together (hpccg_batch_solve_host), each to --rel-tol; SPEC is a list
// "nx,ny,nz/nx,ny,nz/..." or "random:COUNT,LO,HI,SEED" (each of nx, ny, nz
// uniform in [LO, HI] from the project's generator, as the bench's batch).
// --ranks P runs the reference's multi-rank problem (what `mpirun -np P` runs):
// rank q owns the z slab q of the nx x ny x (nz P) grid (SparseMatrix.F90:68-185),
// make_local_matrix's halo plan in the MPI form or, with --halo get, the CAF-V2
// block form, and the reference's CG with rank-order dot sums; all P ranks run
// in this process on the current GPU (hpccg_slab_group_cg_host), with the
// report lines of the reference's rank 0.
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

// The project's counter-based generator (splitmix64 finaliser of
// seed + (i+1) * 0x9E3779B97F4A7C15), the sequence hpccg_gpu_uniform_pm1 draws.
static uint64_t splitmix64_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Grid sizes of a --batch SPEC (see the header); false on a malformed spec.
static bool batch_spec(const char *spec, std::vector<int32_t> *sizes) {
  sizes->clear();
  if (!strncmp(spec, "random:", 7)) {
    long long count = 0, lo = 0, hi = 0, seed = 0;
    if (sscanf(spec + 7, "%lld,%lld,%lld,%lld", &count, &lo, &hi, &seed) != 4 || count < 1 || lo < 1 || hi < lo)
      return false;
    for (long long i = 0; i < 3 * count; ++i)
      sizes->push_back((int32_t)(lo + (long long)(splitmix64_at((uint64_t)seed, (uint64_t)i) % (uint64_t)(hi - lo + 1))));
    return true;
  }
  const char *q = spec;
  while (*q) {
    int a = 0, b = 0, c = 0, used = 0;
    if (sscanf(q, "%d,%d,%d%n", &a, &b, &c, &used) != 3 || a < 1 || b < 1 || c < 1) return false;
    sizes->push_back(a);
    sizes->push_back(b);
    sizes->push_back(c);
    q += used;
    if (*q == '/') ++q;
    else if (*q) return false;
  }
  return !sizes->empty();
}

// b = 27 - (nnzrow - 1) of generate_matrix's row (SparseMatrix.F90:170-172),
// nnzrow the row's kept neighbours; rows in the reference's order, x fastest.
static void reference_rhs(int nx, int ny, int nz, double *b) {
  auto kept = [](int i, int m) { return 1 + (i > 1) + (i < m); };
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t r = 0; r < n; ++r) {
    const int ix = (int)(r % nx) + 1, iy = (int)((r / nx) % ny) + 1, iz = (int)(r / ((int64_t)nx * ny)) + 1;
    b[r] = 27.0 - (double)(kept(ix, nx) * kept(iy, ny) * kept(iz, nz) - 1);
  }
}

static int precision_code(const char *name) {
  if (!strcmp(name, "fp64")) return HPCCG_PREC_FP64;
  if (!strcmp(name, "fp32")) return HPCCG_PREC_FP32;
  if (!strcmp(name, "bf16")) return HPCCG_PREC_BF16;
  return -1;
}
static const char *precision_name(int p) { return p == HPCCG_PREC_FP32 ? "FP32" : p == HPCCG_PREC_BF16 ? "BF16" : "FP64"; }

// --batch: every system of the spec, solved together on the device.
static int run_batch(const std::vector<int32_t> &sizes, int precision, double rel_tol, int max_iter, int spmv_kind,
                     int timing_level) {
  const int nsys = (int)(sizes.size() / 3);
  hpccg_batch *B = nullptr;
  check(hpccg_batch_create_generated(nsys, sizes.data(), &B), "batch_create_generated");
  if (spmv_kind == HPCCG_SPMV_STENCIL) check(hpccg_batch_set_spmv(B, HPCCG_SPMV_STENCIL), "batch_set_spmv");
  int32_t ns = 0;
  int64_t rows = 0;
  check(hpccg_batch_info(B, &ns, &rows, nullptr), "batch_info");
  std::vector<int64_t> offs(2 * (size_t)nsys);
  check(hpccg_batch_info(B, nullptr, nullptr, offs.data()), "batch_info");
  std::vector<double> b((size_t)rows, 0.0), x((size_t)rows, 0.0);
  int64_t total = 0;
  for (int s = 0; s < nsys; ++s) {
    reference_rhs(sizes[3 * s], sizes[3 * s + 1], sizes[3 * s + 2], b.data() + offs[2 * s]);
    total += offs[2 * s + 1];
  }
  printf(" HPCCG Benchmark\n");
  printf(" Using double precision\n");
  printf(" Batch of %d systems, %lld rows in all\n", nsys, (long long)total);
  printf(" Solver: %s\n", precision == HPCCG_PREC_FP64 ? "FP64 CG per system"
                                                      : precision == HPCCG_PREC_FP32
                                                            ? "FP64 iterative refinement, FP32 inner CG per system"
                                                            : "FP64 iterative refinement, BF16-value inner CG per system");
  std::vector<int32_t> iters(nsys), outer(nsys);
  std::vector<double> relres(nsys);
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = hpccg_batch_solve_host(B, b.data(), x.data(), precision, rel_tol, max_iter, iters.data(),
                                        relres.data(), outer.data());
  const auto t1 = std::chrono::steady_clock::now();
  if (rc != HPCCG_OK && rc != HPCCG_ERR_NOT_CONVERGED) check(rc, "batch_solve_host");
  for (int s = 0; s < nsys; ++s) {
    double err = 0.0;
    for (int64_t i = 0; i < offs[2 * s + 1]; ++i) err = std::fmax(err, std::fabs(x[offs[2 * s] + i] - 1.0));
    printf(" System %d (%d x %d x %d): iterations %d, refinement cycles %d, FP64 rel-res %.6e, "
           "max|x - xexact| %.3e\n",
           s, sizes[3 * s], sizes[3 * s + 1], sizes[3 * s + 2], iters[s], outer[s], relres[s], err);
  }
  float ms = 0.f;
  check(hpccg_batch_last_solve_ms(B, &ms), "batch_last_solve_ms");
  if (timing_level > 0) {
    printf(" TIMER: Total %15.7g sec\n", std::chrono::duration<double>(t1 - t0).count());
    printf(" TIMER: Device %15.7g sec\n", 1e-3 * ms);
  }
  if (rc == HPCCG_ERR_NOT_CONVERGED) printf(" Not every system reached the target\n");
  hpccg_batch_destroy(B);
  return rc == HPCCG_OK ? 0 : 3;
}

// --ranks: the reference's P-rank run, all ranks in this process.
static int run_ranks(int nx, int ny, int nz, int nranks, int halo, int max_iter, double tolerance, bool quiet,
                     int timing_level) {
  const int64_t local = (int64_t)nx * ny * nz;
  std::vector<std::vector<int32_t>> rows(nranks), cols(nranks);
  std::vector<std::vector<double>> vals(nranks), x(nranks), b(nranks), xe(nranks);
  std::vector<int64_t> nnz(nranks);
  std::vector<int32_t> first((size_t)nranks + 1);
  for (int q = 0; q <= nranks; ++q) first[q] = (int32_t)(local * q + 1);
  std::vector<hpccg_slab_plan *> plans(nranks, nullptr);
  int64_t total_nnz = 0;
  for (int q = 0; q < nranks; ++q) {
    rows[q].resize(local + 1);
    cols[q].resize(27 * local);
    vals[q].resize(27 * local);
    x[q].resize(local);
    b[q].resize(local);
    xe[q].resize(local);
    check(hpccg_generate_matrix_rank(nx, ny, nz, q, nranks, rows[q].data(), cols[q].data(), vals[q].data(),
                                     x[q].data(), b[q].data(), xe[q].data(), &nnz[q]),
          "generate_matrix_rank");
    total_nnz += nnz[q];
    check(hpccg_slab_plan_create((int32_t)local, nnz[q], rows[q].data(), cols[q].data(), nranks, q, first.data(),
                                 halo, &plans[q]),
          "slab_plan_create");
  }
  if (halo == HPCCG_HALO_MPI) {
    // make_local_matrix's messages (SparseMatrix.F90:563-604): each rank learns, from every
    // neighbour, the global ids that neighbour needs from it, in the neighbour's order
    std::vector<std::vector<int32_t>> nbr(nranks), ext(nranks), own(nranks);
    for (int q = 0; q < nranks; ++q) {
      int32_t ne = 0, nn = 0, nb = 0, ts = 0;
      check(hpccg_slab_plan_info(plans[q], &ne, &nn, &nb, &ts), "slab_plan_info");
      nbr[q].resize(nn);
      std::vector<int32_t> rl(nn);
      check(hpccg_slab_plan_neighbors(plans[q], nbr[q].data(), rl.data()), "slab_plan_neighbors");
      ext[q].resize(ne);
      own[q].resize(ne);
      check(hpccg_slab_plan_externals(plans[q], ext[q].data(), own[q].data()), "slab_plan_externals");
    }
    for (int q = 0; q < nranks; ++q) {
      std::vector<int32_t> lens, ids;
      for (int32_t n : nbr[q]) {
        int32_t cnt = 0;
        for (size_t i = 0; i < ext[n].size(); ++i)
          if (own[n][i] == q) {
            ids.push_back(ext[n][i]);
            ++cnt;
          }
        lens.push_back(cnt);
      }
      static const int32_t none = 0;  // a non-null pointer for an empty list
      check(hpccg_slab_plan_set_sends(plans[q], lens.empty() ? &none : lens.data(), ids.empty() ? &none : ids.data()),
            "slab_plan_set_sends");
    }
  }
  std::vector<hpccg_slab *> slabs(nranks, nullptr);
  for (int q = 0; q < nranks; ++q) check(hpccg_slab_create(plans[q], vals[q].data(), &slabs[q]), "slab_create");

  // printInfo of the reference's rank 0 (main.F90:58-71): total_nrow = P local_nrow, total_nnz = 27 total_nrow
  printf(" HPCCG Benchmark\n");
  printf(" Using double precision\n");
  printf(" Total size (N x N): %12lld\n", (long long)(local * nranks));
  printf(" Total nonzeroes: %12lld\n", (long long)(27 * local * nranks));
  printf(" Ranks: %d z slabs in one process (halo %s), stored nonzeroes %lld\n", nranks,
         halo == HPCCG_HALO_MPI ? "MPI send lists" : "CAF-V2 block gets", (long long)total_nnz);
  printf(" OpenMP disabled.\n");
  std::vector<const double *> bp(nranks);
  std::vector<double *> xp(nranks);
  for (int q = 0; q < nranks; ++q) {
    bp[q] = b[q].data();
    xp[q] = x[q].data();
  }
  std::vector<double> hist((size_t)max_iter + 1);
  int32_t niters = 0;
  double normr = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = hpccg_slab_group_cg_host(slabs.data(), nranks, bp.data(), xp.data(), max_iter, tolerance, &niters,
                                          &normr, hist.data());
  const auto t1 = std::chrono::steady_clock::now();
  if (rc != HPCCG_OK && rc != HPCCG_ERR_BREAKDOWN) check(rc, "slab_group_cg");
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
  if (timing_level > 0) printf(" TIMER: Total %15.7g sec\n", std::chrono::duration<double>(t1 - t0).count());
  double err = 0.0;
  for (int q = 0; q < nranks; ++q)
    for (int64_t i = 0; i < local; ++i) err = std::fmax(err, std::fabs(x[q][i] - xe[q][i]));
  printf(" Iterations: %d  final normr: %.17g  max|x - xexact|: %.3e\n", niters, normr, err);
  for (int q = 0; q < nranks; ++q) {
    hpccg_slab_destroy(slabs[q]);
    hpccg_slab_plan_destroy(plans[q]);
  }
  return rc == HPCCG_OK ? 0 : 3;
}

int main(int argc, char **argv) {
  int max_iter = 150;    // main.F90:127
  double tolerance = 0;  // main.F90:128
  double rel_tol = 1e-8;
  bool device_generate = false, quiet = false;
  int timing_level = 1;  // MPI/config.mk TIMER_LEVEL
  int spmv_kind = HPCCG_SPMV_AUTO, spmv_param = 0;
  int precision = HPCCG_PREC_FP64;
  int nranks = 0, halo = HPCCG_HALO_MPI;
  const char *batch = nullptr;
  std::vector<int> pos;
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--max-iter") && i + 1 < argc) max_iter = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--tol") && i + 1 < argc) tolerance = atof(argv[++i]);
    else if (!strcmp(argv[i], "--rel-tol") && i + 1 < argc) rel_tol = atof(argv[++i]);
    else if (!strcmp(argv[i], "--device-generate")) device_generate = true;
    else if (!strcmp(argv[i], "--quiet")) quiet = true;
    else if (!strcmp(argv[i], "--timing-level") && i + 1 < argc) timing_level = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--batch") && i + 1 < argc) batch = argv[++i];
    else if (!strcmp(argv[i], "--ranks") && i + 1 < argc) {
      nranks = atoi(argv[++i]);
      if (nranks < 1) {
        fprintf(stderr, "HPCCG-B200: --ranks must be positive\n");
        return 2;
      }
    } else if (!strcmp(argv[i], "--halo") && i + 1 < argc) {
      ++i;
      if (!strcmp(argv[i], "mpi")) halo = HPCCG_HALO_MPI;
      else if (!strcmp(argv[i], "get")) halo = HPCCG_HALO_GET;
      else {
        fprintf(stderr, "HPCCG-B200: --halo takes mpi or get\n");
        return 2;
      }
    }
    else if (!strcmp(argv[i], "--precision") && i + 1 < argc) {
      precision = precision_code(argv[++i]);
      if (precision < 0) {
        fprintf(stderr, "HPCCG-B200: --precision takes fp64, fp32 or bf16\n");
        return 2;
      }
    } else if (!strcmp(argv[i], "--spmv") && i + 1 < argc) {
      spmv_kind = atoi(argv[++i]);
      const char *comma = strchr(argv[i], ',');
      if (comma) spmv_param = atoi(comma + 1);
    } else if (argv[i][0] != '-' && pos.size() < 3) {
      pos.push_back(atoi(argv[i]));
    } else {
      fprintf(stderr, "HPCCG-B200: unknown option %s\n", argv[i]);
      return 2;
    }
  }
  if (!(rel_tol > 0.0)) {
    fprintf(stderr, "HPCCG-B200: --rel-tol must be positive\n");
    return 2;
  }
  if (batch) {
    std::vector<int32_t> sizes;
    if (!batch_spec(batch, &sizes)) {
      fprintf(stderr, "HPCCG-B200: bad --batch spec %s\n", batch);
      return 2;
    }
    return run_batch(sizes, precision, rel_tol, max_iter, spmv_kind, timing_level);
  }
  if (pos.size() < 3) {
    printf(" USAGE: ./HPCCG <nx> <ny> <nz>\n");
    return 0;
  }
  const int nx = pos[0], ny = pos[1], nz = pos[2];
  if (nx < 1 || ny < 1 || nz < 1) {
    fprintf(stderr, "HPCCG-B200: nx, ny, nz must be positive\n");
    return 2;
  }
  if (nranks > 0) return run_ranks(nx, ny, nz, nranks, halo, max_iter, tolerance, quiet, timing_level);
  const int64_t n = (int64_t)nx * ny * nz;
  std::vector<double> x(n), b(n), xexact(n);
  hpccg_ctx *ctx = nullptr;
  int64_t nnz = 0;
  if (device_generate) {
    // A is built on the device; x0, b and xexact follow from the row's kept
    // neighbour count, b = 27 - (nnzrow - 1) (SparseMatrix.F90:170-172).
    check(hpccg_gpu_create_generated(nx, ny, nz, nullptr, nullptr, nullptr, &ctx), "generate");
    check(hpccg_gpu_info(ctx, nullptr, &nnz, nullptr), "info");
    reference_rhs(nx, ny, nz, b.data());
    for (int64_t r = 0; r < n; ++r) {
      x[r] = 0.0;
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

  if (precision != HPCCG_PREC_FP64) {
    // FP64 iterative refinement around the low-precision inner CG, to rel_tol
    printf(" Solver: FP64 iterative refinement, %s inner CG, FP64 rel-res target %g\n", precision_name(precision),
           rel_tol);
    hpccg_mixed_info info{};
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = hpccg_gpu_solve_mixed(ctx, b.data(), x.data(), precision, rel_tol, 30, max_iter, 0.0, &info);
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != HPCCG_OK && rc != HPCCG_ERR_NOT_CONVERGED) check(rc, "solve_mixed");
    printf(" Refinement cycles: %d  inner iterations: %d  FP64 rel-res: %.6e\n", info.outer_iters, info.inner_iters,
           info.relres);
    float solve_ms = 0.f;
    check(hpccg_gpu_last_solve_ms(ctx, &solve_ms), "last_solve_ms");
    if (timing_level > 0) {
      printf(" TIMER: Total %15.7g sec\n", std::chrono::duration<double>(t1 - t0).count());
      printf(" TIMER: Device %15.7g sec\n", 1e-3 * solve_ms);
    }
    double err = 0.0;
    for (int64_t i = 0; i < n; ++i) err = std::fmax(err, std::fabs(x[i] - xexact[i]));
    printf(" max|x - xexact|: %.3e\n", err);
    if (rc == HPCCG_ERR_NOT_CONVERGED) printf(" Not converged in 30 refinement cycles\n");
    hpccg_gpu_destroy(ctx);
    return rc == HPCCG_OK ? 0 : 3;
  }

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
