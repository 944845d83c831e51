// perman_cli.cpp -- drop-in `perman` command line over libperman_b200.so.
//
// Mirrors the reference CLI (main.cu:315-590): the same flags and algorithm
// ids, the same input format, the same "Result: <name> <value> in <seconds>"
// line (printed with 17 significant digits instead of cout's 6).
//   -m FILE | -f FILE   matrix file (the README documents -m, main.cu reads -f)
//   -p ID               algorithm id (default 1)
//   -s                  sparse algorithms        -b   binary (every entry 1)
//   -a                  approximation            -x N trials (default 100000)
//   -y N                scale interval (4)       -z N scale sweeps (5)
//   -r N                preprocessing: 0 none, 1 sortOrder, 2 skipOrder
//   -g                  GPU (the default)        -d N GPUs for multi-GPU ids (2)
//   -t N                accepted, unused (host threads of the CPU algorithms)
//   -c                  CPU algorithms: not part of this engine -> error
//   --seed N            Monte-Carlo seed (default: time, like the reference)
//   -i -m M -n N        grid-graph mode (main.cu:250-313): approximate
//                       permanent of the M x N board's grid graph (domino
//                       tilings); with -i, -m and -n are the board sides.
#include <getopt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "perman_b200.h"

namespace {

struct Options {
  std::string file, m_arg;
  int gridn = 36;
  bool binary = false, sparse = false, approx = false, cpu = false, gpu = false, grid = false;
  int algo = 1, threads = 16, gpu_num = 2, pre = 0;
  int times = 100000, y = 4, z = 5;
  long long seed = -1;
};

int usage(const char* msg) {
  fprintf(stderr, "%s\n", msg);
  return 1;
}

double now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// The engine kernel that produced an exact result (perm_result.kernel).
const char* kernel_name(int k) {
  switch (k) {
    case PERM_KERNEL_DENSE: return "FP64-X walk";
    case PERM_KERNEL_SKIPPER: return "SkipPer";
    case PERM_KERNEL_DENSE_INT: return "int32-X walk";
    case PERM_KERNEL_DENSE_DD: return "double-double walk";
    case PERM_KERNEL_DENSE_TC: return "tensor-core row sums";
    case PERM_KERNEL_DENSE_SPLIT: return "split-X walk";
    case PERM_KERNEL_DENSE_INT_DD: return "int32-X walk, double-double products and sum";
    case PERM_KERNEL_DENSE_SDD: return "split-dd walk";
    default: return "unknown";
  }
}

void print_result(const char* name, double value, double seconds) {
  printf("Result: %s %.17g in %.6f\n", name, value, seconds);
  fflush(stdout);
}

int die(perm_ctx* ctx, int rc) {
  fprintf(stderr, "perman: %s: %s\n", perm_status_string(rc), ctx ? perm_ctx_last_error(ctx) : "");
  return 3;
}

// Multi-GPU exact: perm_exact_dense_multi (one host thread and context per
// device, shards of the Gray range walked by `variant` -- 0: the engine's
// choice per shard -- and a double-double sum of the per-device results).
// Evaluates once, like the reference's multi-GPU ids (no error estimate on
// the sum).
int multi_gpu_dense(const std::vector<double>& a, int n, int gpus, int variant, perm_result* total) {
  int avail = perm_device_count();
  if (avail < 1) {
    fprintf(stderr, "perman: no CUDA device\n");
    return 3;
  }
  gpus = std::max(1, std::min(gpus, avail));
  const int rc = perm_exact_dense_multi(a.data(), n, PERM_F64, variant, gpus, nullptr, total);
  if (rc != PERM_OK) {
    fprintf(stderr, "perman: %s\n", perm_status_string(rc));
    return 3;
  }
  return 0;
}

// Grid-graph mode: approximate algorithms only, on the board's sparse pattern
// (main.cu:250-313 calls the sparse GPU estimators with grid_graph = true).
int run_grid(const Options& o) {
  const int gm = o.m_arg.empty() ? 36 : atoi(o.m_arg.c_str());
  const int gn = o.gridn;
  if (o.cpu && !o.gpu) return usage("perman: the CPU algorithms (-c) are not part of the B200 engine; run with -g");
  const int nov = gm * gn / 2;
  if (gm < 1 || gn < 1 || nov > PERM_MAX_MC_SPARSE_N) return usage("perman: grid sides out of range");
  std::vector<double> a((size_t)nov * nov);
  int k = 0;
  if (perm_grid_graph(gm, gn, nov, a.data(), &k) != PERM_OK) {
    printf("one of the grid dimensions should be positive.");
    return 0;
  }
  std::vector<int> rptrs(nov + 1, 0), cols, cptrs(nov + 1, 0), rows;
  for (int i = 0; i < nov; i++) {
    for (int j = 0; j < nov; j++)
      if (a[(size_t)i * nov + j] != 0) cols.push_back(j);
    rptrs[i + 1] = (int)cols.size();
  }
  for (int j = 0; j < nov; j++) {
    for (int i = 0; i < nov; i++)
      if (a[(size_t)i * nov + j] != 0) rows.push_back(i);
    cptrs[j + 1] = (int)rows.size();
  }
  static const char* names[] = {nullptr, "gpu_perman64_rasmussen_sparse", "gpu_perman64_approximation_sparse",
                                "gpu_perman64_rasmussen_multigpucpu_chunks",
                                "gpu_perman64_approximation_multigpucpu_chunks_sparse"};
  if (o.algo < 1 || o.algo > 4) {
    printf("Unknown Algorithm ID\n");
    return 0;
  }
  perm_ctx* ctx = nullptr;
  const double t0 = now();
  int rc = perm_ctx_create(0, &ctx);
  if (rc != PERM_OK) {
    fprintf(stderr, "perman: cannot use a B200: %s\n", perm_status_string(rc));
    return 3;
  }
  perm_estimate e;
  const bool scaling = o.algo == 2 || o.algo == 4;
  rc = scaling ? perm_approx_scaling_sparse(ctx, nov, rptrs.data(), cols.data(), cptrs.data(), rows.data(), o.times,
                                            o.y, o.z, (uint64_t)o.seed, nullptr, &e)
               : perm_approx_rasmussen_sparse(ctx, nov, rptrs.data(), cols.data(), o.times, (uint64_t)o.seed,
                                              nullptr, &e);
  int status = 0;
  if (rc != PERM_OK) {
    status = die(ctx, rc);
  } else {
    printf("kernel in %.6f\n", e.kernel_ms * 1e-3);
    printf("number of zeros: %.0f\n", e.zero_trials);
    printf("std error: %.17g (%.0f trials, seed %lld)\n", e.std_error, e.trials, o.seed);
    print_result(names[o.algo], e.mean, now() - t0);
  }
  perm_ctx_destroy(ctx);
  return status;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  const char* short_opts = "bsr:t:f:gd:cap:x:y:z:im:n:";
  const struct option long_opts[] = {
      {"binary", 0, nullptr, 'b'},         {"sparse", 0, nullptr, 's'},
      {"preprocessing", 1, nullptr, 'r'},  {"threads", 1, nullptr, 't'},
      {"file", 1, nullptr, 'f'},           {"gpu", 0, nullptr, 'g'},
      {"device", 1, nullptr, 'd'},         {"cpu", 0, nullptr, 'c'},
      {"approximation", 0, nullptr, 'a'},  {"perman", 1, nullptr, 'p'},
      {"numOfTimes", 1, nullptr, 'x'},     {"scaleIntervals", 1, nullptr, 'y'},
      {"scaleTimes", 1, nullptr, 'z'},     {"grid", 0, nullptr, 'i'},
      {"matrix", 1, nullptr, 'm'},         {"gridn", 1, nullptr, 'n'},
      {"seed", 1, nullptr, 'S'},           {nullptr, 0, nullptr, 0}};
  int c;
  while ((c = getopt_long(argc, argv, short_opts, long_opts, nullptr)) != -1) {
    if (optarg && optarg[0] == '-' && c != 'S') {
      fprintf(stderr, "Option -%c requires an argument.\n", c);
      return 1;
    }
    switch (c) {
      case 'b': o.binary = true; break;
      case 's': o.sparse = true; break;
      case 'r': o.pre = atoi(optarg); break;
      case 't': o.threads = atoi(optarg); break;
      case 'f': o.file = optarg; break;
      case 'm': o.m_arg = optarg; break;
      case 'g': o.gpu = true; break;
      case 'd': o.gpu_num = atoi(optarg); break;
      case 'c': o.cpu = true; break;
      case 'a': o.approx = true; break;
      case 'p': o.algo = atoi(optarg); break;
      case 'x': o.times = atoi(optarg); break;
      case 'y': o.y = atoi(optarg); break;
      case 'z': o.z = atoi(optarg); break;
      case 'i': o.grid = true; break;
      case 'n': o.gridn = atoi(optarg); break;
      case 'S': o.seed = atoll(optarg); break;
      default: return 1;
    }
  }
  for (int i = optind; i < argc; i++) printf("Non-option argument %s\n", argv[i]);
  if (o.seed < 0) o.seed = (long long)time(nullptr);
  if (!o.grid && o.file.empty()) o.file = o.m_arg;
  if (o.grid) return run_grid(o);
  if (o.file.empty()) return usage("Option -f (or -m) is a required argument.");
  if (o.cpu && !o.gpu)
    return usage("perman: the CPU algorithms (-c) are not part of the B200 engine; run with -g");
  if (o.pre < 0 || o.pre > 2) return usage("perman: -r must be 0, 1 or 2");
  if (o.seed < 0) o.seed = (long long)time(nullptr);

  // read header first to size the buffer
  FILE* fh = fopen(o.file.c_str(), "r");
  if (!fh) {
    fprintf(stderr, "perman: cannot open '%s'\n", o.file.c_str());
    return 1;
  }
  int hn = 0;
  if (fscanf(fh, "%d", &hn) != 1 || hn <= 0 || hn > 4096) {
    fclose(fh);
    fprintf(stderr, "perman: bad header in '%s'\n", o.file.c_str());
    return 1;
  }
  fclose(fh);
  std::vector<double> a((size_t)hn * hn);
  int n = 0, hnnz = 0;
  char type[8] = {0};
  int rc = perm_read_matrix(o.file.c_str(), o.binary, hn, a.data(), &n, &hnnz, type);
  if (rc != PERM_OK) return 1;
  a.resize((size_t)n * n);
  std::vector<int> cptrs(n + 1), rptrs(n + 1), rows((size_t)n * n), cols((size_t)n * n);
  std::vector<double> cvals((size_t)n * n), rvals((size_t)n * n);
  int nnz = perm_compress(o.pre, a.data(), n, cptrs.data(), rows.data(), cvals.data(), rptrs.data(), cols.data(),
                          rvals.data());
  if (nnz < 0) return usage("perman: compression failed");

  perm_ctx* ctx = nullptr;
  const double t0 = now();
  rc = perm_ctx_create(0, &ctx);
  if (rc != PERM_OK) {
    fprintf(stderr, "perman: cannot use a B200: %s\n", perm_status_string(rc));
    return 3;
  }
  int status = 0;
  if (!o.approx) {
    perm_result r;
    const char* name = nullptr;
    if (!o.sparse) {
      static const char* names[] = {"gpu_perman64_xlocal", "gpu_perman64_xlocal", "gpu_perman64_xshared",
                                    "gpu_perman64_xshared_coalescing",
                                    "gpu_perman64_xshared_coalescing_mshared"};
      if (o.algo >= 0 && o.algo <= 4) {
        name = names[o.algo];
        rc = perm_exact_dense(ctx, a.data(), n, PERM_F64, &r);
      } else if (o.algo == 5 || o.algo == 6 || o.algo == 66) {
        name = o.algo == 5   ? "gpu_perman64_xshared_coalescing_mshared_multigpu"
               : o.algo == 6 ? "gpu_perman64_xshared_coalescing_mshared_multigpucpu_chunks"
                             : "gpu_perman64_xshared_coalescing_mshared_multigpu_manual_distribution";
        perm_ctx_destroy(ctx);
        ctx = nullptr;
        if (multi_gpu_dense(a, n, o.algo == 66 ? 4 : o.gpu_num, 0, &r)) return 3;
        rc = PERM_OK;
      } else {
        printf("Unknown Algorithm ID\n");
        perm_ctx_destroy(ctx);
        return 0;
      }
    } else {
      static const char* snames[] = {nullptr,
                                     "gpu_perman64_xlocal_sparse",
                                     "gpu_perman64_xshared_sparse",
                                     "gpu_perman64_xshared_coalescing_sparse",
                                     "gpu_perman64_xshared_coalescing_mshared_sparse",
                                     "gpu_perman64_xshared_coalescing_mshared_multigpu_sparse",
                                     "gpu_perman64_xshared_coalescing_mshared_multigpucpu_chunks_sparse",
                                     "gpu_perman64_xshared_coalescing_mshared_skipper",
                                     "gpu_perman64_xshared_coalescing_mshared_multigpucpu_chunks_skipper"};
      if ((o.algo >= 1 && o.algo <= 8) || o.algo == 66) {
        name = o.algo == 66 ? "gpu_perman64_xshared_coalescing_mshared_multigpu_sparse_manual_distribution"
                            : snames[o.algo];
        // -p1..-p6 and -p66 are the reference's CCS walks that touch only the
        // flipped column's nonzeros (gpu_exact_sparse.cu:194-552; -p5, -p6,
        // -p66 on several devices, :823-1120): here the split-dd kernel,
        // whose sparse layout walks only the rows of the three sparsest
        // columns at seven of eight steps (orders 4..40), sharded over -d
        // devices for the multi-GPU ids; -p7/-p8 and matrices outside the
        // split-dd orders run the sparse dispatcher (SkipPer when most terms
        // vanish)
        const bool sdd = perm_sdd_layout(a.data(), n) >= 0;
        const bool multi = o.algo == 5 || o.algo == 6 || o.algo == 66;
        if (multi && sdd) {
          perm_ctx_destroy(ctx);
          ctx = nullptr;
          if (multi_gpu_dense(a, n, o.algo == 66 ? 4 : o.gpu_num, PERM_KERNEL_DENSE_SDD, &r)) return 3;
          rc = PERM_OK;
        } else {
          const bool ccs_walk = o.algo >= 1 && o.algo <= 4 && sdd;
          rc = perm_exact_sparse_ex(ctx, n, rptrs.data(), cols.data(), rvals.data(), cptrs.data(), rows.data(),
                                    cvals.data(), ccs_walk ? PERM_KERNEL_DENSE_SDD : 0, &r);
        }
      } else {
        printf("Unknown Algorithm ID\n");
        perm_ctx_destroy(ctx);
        return 0;
      }
    }
    if (rc != PERM_OK) {
      status = die(ctx, rc);
    } else {
      printf("kernel in %.6f\n", r.kernel_ms * 1e-3);
      printf("engine kernel: %s\n", kernel_name(r.kernel));
      print_result(name, r.value, now() - t0);
    }
  } else {
    perm_estimate e;
    const char* name = nullptr;
    bool scaling = (o.algo == 2 || o.algo == 4);
    if (o.algo < 1 || o.algo > 4) {
      printf("Unknown Algorithm ID\n");
      perm_ctx_destroy(ctx);
      return 0;
    }
    if (!o.sparse) {
      static const char* names[] = {nullptr, "gpu_perman64_rasmussen", "gpu_perman64_approximation",
                                    "gpu_perman64_rasmussen_multigpucpu_chunks",
                                    "gpu_perman64_approximation_multigpucpu_chunks"};
      name = names[o.algo];
      rc = scaling ? perm_approx_scaling(ctx, a.data(), n, PERM_F64, o.times, o.y, o.z, (uint64_t)o.seed, nullptr, &e)
                   : perm_approx_rasmussen(ctx, a.data(), n, PERM_F64, o.times, (uint64_t)o.seed, nullptr, &e);
    } else {
      static const char* names[] = {nullptr, "gpu_perman64_rasmussen_sparse", "gpu_perman64_approximation_sparse",
                                    "gpu_perman64_rasmussen_multigpucpu_chunks_sparse",
                                    "gpu_perman64_approximation_multigpucpu_chunks_sparse"};
      name = names[o.algo];
      rc = scaling ? perm_approx_scaling_sparse(ctx, n, rptrs.data(), cols.data(), cptrs.data(), rows.data(), o.times,
                                                o.y, o.z, (uint64_t)o.seed, nullptr, &e)
                   : perm_approx_rasmussen_sparse(ctx, n, rptrs.data(), cols.data(), o.times, (uint64_t)o.seed,
                                                  nullptr, &e);
    }
    if (rc != PERM_OK) {
      status = die(ctx, rc);
    } else {
      printf("kernel in %.6f\n", e.kernel_ms * 1e-3);
      printf("number of zeros: %.0f\n", e.zero_trials);
      printf("std error: %.17g (%.0f trials, seed %lld)\n", e.std_error, e.trials, o.seed);
      print_result(name, e.mean, now() - t0);
    }
  }
  perm_ctx_destroy(ctx);
  return status;
}
