// ref_harness.cu -- TEST INFRASTRUCTURE ONLY.
//
// Builds the reference implementation (berkyaglioglu/matrix-permanent-calculator)
// from its own, unmodified source files into oracle/_ref/libperman_ref.so so that
// tests and the CPU-baseline leg of bench.py can call the reference functions
// directly, at full double precision (the reference CLI prints 6 digits only).
//
// Nothing here is product code: only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / --impl reference legs load this library.
//
// The reference's main.cu textually includes util.h, algo.h and the four .cu
// files (main.cu:9-15); its main() is renamed so that the library has none.
// Recipe: oracle/build_ref.sh (reads the sources where they lie).

#define main perman_reference_cli_main
#include "main.cu"
#undef main

#include <cstring>

namespace {

template <class T>
T* copy_mat(const T* src, int n) {
  T* m = new T[(size_t)n * n];
  std::memcpy(m, src, sizeof(T) * (size_t)n * n);
  return m;
}

// Ownership shim: the reference compressors allocate with new[]; hand the
// arrays back through caller buffers and free them here.
template <class T>
int compress_into(int mode, T* mat, int nov, int nnz, int* cptrs, int* rows, T* cvals,
                  int* rptrs, int* cols, T* rvals) {
  int *cp, *rw, *rp, *cl;
  T *cv, *rv;
  if (mode == 1) {
    matrix2compressed_sortOrder(mat, cp, rw, cv, rp, cl, rv, nov, nnz);   // util.h:554
  } else if (mode == 2) {
    matrix2compressed_skipOrder(mat, cp, rw, cv, rp, cl, rv, nov, nnz);   // util.h:622
  } else {
    matrix2compressed(mat, cp, rw, cv, rp, cl, rv, nov, nnz);             // util.h:523
  }
  int used = rp[nov];
  std::memcpy(cptrs, cp, sizeof(int) * (nov + 1));
  std::memcpy(rptrs, rp, sizeof(int) * (nov + 1));
  std::memcpy(rows, rw, sizeof(int) * used);
  std::memcpy(cols, cl, sizeof(int) * used);
  std::memcpy(cvals, cv, sizeof(T) * used);
  std::memcpy(rvals, rv, sizeof(T) * used);
  delete[] cp; delete[] rw; delete[] cv; delete[] rp; delete[] cl; delete[] rv;
  return used;
}

}  // namespace

extern "C" {

// ---- matrix I/O and preprocessing (util.h) -------------------------------
// Reads a reference-format file with the reference reader (util.h:344) into a
// caller-zeroed n*n buffer.  Returns n, or -1 on open failure.
int ref_read_matrix_f64(const char* path, int generic, double* out, int cap_n, int* nnz_out) {
  std::ifstream in(path);
  if (!in) return -1;
  std::string line;
  std::getline(in, line);
  std::istringstream iss(line);
  int nov, nnz; std::string type;
  iss >> nov >> nnz >> type;
  if (nov > cap_n) return -2;
  if (nnz_out) *nnz_out = nnz;
  if (type == "int") {
    int* m = new int[(size_t)nov * nov]();
    ReadMatrix(m, in, nov, generic != 0);
    for (int i = 0; i < nov * nov; i++) out[i] = m[i];
    delete[] m;
  } else if (type == "float") {
    float* m = new float[(size_t)nov * nov]();
    ReadMatrix(m, in, nov, generic != 0);
    for (int i = 0; i < nov * nov; i++) out[i] = m[i];
    delete[] m;
  } else {
    double* m = new double[(size_t)nov * nov]();
    ReadMatrix(m, in, nov, generic != 0);
    for (int i = 0; i < nov * nov; i++) out[i] = m[i];
    delete[] m;
  }
  return nov;
}

// mode 0: matrix2compressed, 1: sortOrder, 2: skipOrder.  `mat` is permuted in
// place for modes 1 and 2 exactly as the reference does.  Returns the number
// of stored (> 0) entries.
int ref_compress_f64(int mode, double* mat, int nov, int nnz, int* cptrs, int* rows, double* cvals,
                     int* rptrs, int* cols, double* rvals) {
  return compress_into<double>(mode, mat, nov, nnz, cptrs, rows, cvals, rptrs, cols, rvals);
}

// Grid-graph matrix (util.h:403-520) into a caller buffer of cap x cap
// doubles; returns nov or <0.
int ref_grid_graph(int m, int n, double* out, int cap) {
  int *mat, *cptrs, *rows, *rptrs, *cols;
  int nnz = gridGraph2compressed(m, n, mat, cptrs, rows, rptrs, cols);
  if (nnz == -1) return -1;
  const int nov = m * n / 2;
  int rc = nov;
  if (nov > cap) rc = -2;
  else
    for (int i = 0; i < nov * nov; i++) out[i] = mat[i];
  delete[] mat;
  delete[] cptrs;
  delete[] rows;
  delete[] rptrs;
  delete[] cols;
  return rc;
}

// ---- CPU exact (algo.h) ----------------------------------------------------
double ref_parallel_perman64_f64(const double* mat, int nov, int threads) {   // algo.h:663
  double* m = copy_mat(mat, nov);
  double r = parallel_perman64(m, nov, threads);
  delete[] m;
  return r;
}
double ref_parallel_perman64_i32(const int* mat, int nov, int threads) {
  int* m = copy_mat(mat, nov);
  double r = parallel_perman64(m, nov, threads);
  delete[] m;
  return r;
}
double ref_perman64_f64(const double* mat, int nov) {                            // algo.h:1032
  double* m = copy_mat(mat, nov);
  double r = perman64(m, nov);
  delete[] m;
  return r;
}
double ref_parallel_perman64_sparse_f64(const double* mat, const int* cptrs, const int* rows,
                                        const double* cvals, int nov, int threads) {  // algo.h:569
  double* m = copy_mat(mat, nov);
  double r = parallel_perman64_sparse(m, (int*)cptrs, (int*)rows, (double*)cvals, nov, threads);
  delete[] m;
  return r;
}
double ref_parallel_skip_balanced_f64(const int* rptrs, const int* cols, const double* rvals,
                                      const int* cptrs, const int* rows, const double* cvals,
                                      int nov, int threads) {                   // algo.h:886
  return parallel_skip_perman64_w_balanced((int*)rptrs, (int*)cols, (double*)rvals, (int*)cptrs,
                                           (int*)rows, (double*)cvals, nov, threads);
}

// Range-restricted Ryser sum over Gray indices [start, end), reference
// cpu_perman64 (gpu_exact_dense.cu:7-69) with the x vector and transpose built
// as its hybrid callers build them (gpu_exact_dense.cu:787-800).  Returns the
// raw partial sum (no initial product, no final (4(n&1)-2) factor); used as a
// bounded sample of a large exact workload.
double ref_cpu_perman64_range_f64(const double* mat, int nov, long long start, long long end,
                                  int threads) {
  double* x = new double[nov];
  for (int j = 0; j < nov; j++) {
    double rs = 0;
    for (int k = 0; k < nov; k++) rs += mat[j * nov + k];
    x[j] = mat[j * nov + (nov - 1)] - rs / 2;
  }
  double* mat_t = new double[(size_t)nov * nov];
  for (int i = 0; i < nov; i++)
    for (int j = 0; j < nov; j++) mat_t[i * nov + j] = mat[j * nov + i];
  double r = cpu_perman64(mat_t, x, nov, start, end, threads);
  delete[] x;
  delete[] mat_t;
  return r;
}

// ---- CPU approximate (algo.h) -----------------------------------------------
double ref_rasmussen_f64(const double* mat, int nov, int times, int threads) {  // algo.h:270
  double* m = copy_mat(mat, nov);
  double r = rasmussen(m, nov, times, threads);
  delete[] m;
  return r;
}
double ref_approximation_f64(const double* mat, int nov, int times, int y, int z,
                             int threads) {                                     // algo.h:472
  double* m = copy_mat(mat, nov);
  double r = approximation_perman64(m, nov, times, y, z, threads);
  delete[] m;
  return r;
}
double ref_rasmussen_sparse_f64(const double* mat, const int* rptrs, const int* cols, int nov,
                                int times, int threads) {                       // algo.h:172
  double* m = copy_mat(mat, nov);
  double r = rasmussen_sparse(m, (int*)rptrs, (int*)cols, nov, times, threads);
  delete[] m;
  return r;
}
double ref_approximation_sparse(const int* cptrs, const int* rows, const int* rptrs,
                                const int* cols, int nov, int times, int y, int z,
                                int threads) {                                   // algo.h:366
  return approximation_perman64_sparse((int*)cptrs, (int*)rows, (int*)rptrs, (int*)cols, nov, times,
                                       y, z, threads);
}

// ---- reference GPU wrappers (same-box GPU comparison point) -----------------
double ref_gpu_dense_mshared_f64(const double* mat, int nov, int grid, int block) {  // gpu_exact_dense.cu:641
  double* m = copy_mat(mat, nov);
  double r = gpu_perman64_xshared_coalescing_mshared(m, nov, grid, block);
  delete[] m;
  return r;
}
double ref_gpu_dense_mshared_i32(const int* mat, int nov, int grid, int block) {
  int* m = copy_mat(mat, nov);
  double r = gpu_perman64_xshared_coalescing_mshared(m, nov, grid, block);
  delete[] m;
  return r;
}
double ref_gpu_skipper_f64(const double* mat, const int* rptrs, const int* cols, const int* cptrs,
                           const int* rows, const double* cvals, int nov, int grid,
                           int block) {                                          // gpu_exact_sparse.cu:1124
  double* m = copy_mat(mat, nov);
  double r = gpu_perman64_xshared_coalescing_mshared_skipper(m, (int*)rptrs, (int*)cols, (int*)cptrs,
                                                             (int*)rows, (double*)cvals, nov, grid,
                                                             block);
  delete[] m;
  return r;
}
double ref_gpu_rasmussen_f64(const double* mat, int nov, int times) {          // gpu_approximation_dense.cu:374
  double* m = copy_mat(mat, nov);
  double r = gpu_perman64_rasmussen(m, nov, times);
  delete[] m;
  return r;
}
double ref_gpu_approximation_f64(const double* mat, int nov, int times, int y, int z) {  // :528
  double* m = copy_mat(mat, nov);
  double r = gpu_perman64_approximation(m, nov, times, y, z);
  delete[] m;
  return r;
}

// The reference's GPU wrappers check no CUDA status; this reports (and
// clears) the last error after one of them, as a string.
const char* ref_last_cuda_error() { return cudaGetErrorString(cudaGetLastError()); }

}  // extern "C"
