// matrix_io.cpp -- see matrix_io.h.
#include "matrix_io.h"

#include <algorithm>
#include <climits>
#include <fstream>
#include <sstream>

namespace perm {

namespace {

template <class T>
std::string read_entries(std::istream& in, int n, bool binary, std::vector<double>* a) {
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream iss(line);
    int i, j;
    T val;
    if (!(iss >> i >> j >> val)) continue;  // erroneous line (util.h:351)
    if (i < 0 || j < 0 || i >= n || j >= n) {
      return "entry (" + std::to_string(i) + ", " + std::to_string(j) + ") outside a " +
             std::to_string(n) + "x" + std::to_string(n) + " matrix";
    }
    (*a)[(size_t)i * n + j] = binary ? 1.0 : (double)val;
  }
  return "";
}

}  // namespace

std::string read_matrix_file(const std::string& path, bool binary, HostMatrix* out) {
  std::ifstream in(path);
  if (!in) return "cannot open matrix file '" + path + "'";
  std::string header;
  if (!std::getline(in, header)) return "empty matrix file '" + path + "'";
  std::istringstream hs(header);
  int n = 0, nnz = 0;
  std::string type;
  if (!(hs >> n >> nnz >> type)) return "bad header '" + header + "' (want: n nnz type)";
  if (n <= 0 || n > 4096) return "matrix order " + std::to_string(n) + " outside [1, 4096]";
  out->n = n;
  out->header_nnz = nnz;
  out->type = type;
  out->a.assign((size_t)n * n, 0.0);
  if (type == "int") return read_entries<int>(in, n, binary, &out->a);
  if (type == "float") return read_entries<float>(in, n, binary, &out->a);
  if (type == "double") return read_entries<double>(in, n, binary, &out->a);
  return "unknown value type '" + type + "' (want int, float or double)";
}

void compress(const double* a, int n, Compressed* out) {
  out->n = n;
  out->rptrs.assign(n + 1, 0);
  out->cptrs.assign(n + 1, 0);
  out->cols.clear();
  out->rows.clear();
  out->rvals.clear();
  out->cvals.clear();
  for (int i = 0; i < n; i++) {
    out->rptrs[i] = (int)out->cols.size();
    out->cptrs[i] = (int)out->rows.size();
    for (int j = 0; j < n; j++) {
      double r = a[(size_t)i * n + j];
      if (r > 0) {
        out->cols.push_back(j);
        out->rvals.push_back(r);
      }
      double c = a[(size_t)j * n + i];
      if (c > 0) {
        out->rows.push_back(j);
        out->cvals.push_back(c);
      }
    }
  }
  out->rptrs[n] = (int)out->cols.size();
  out->cptrs[n] = (int)out->rows.size();
}

void compress_sort_order(double* a, int n, Compressed* out) {
  std::vector<std::pair<int, int>> order(n);
  for (int j = 0; j < n; j++) {
    int cnt = 0;
    for (int i = 0; i < n; i++)
      if (a[(size_t)i * n + j] > 0) cnt++;
    order[j] = {j, cnt};
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<int, int>& l, const std::pair<int, int>& r) {
                     return l.second < r.second;
                   });
  std::vector<double> b((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int idx = 0; idx < n; idx++) {
      double v = a[(size_t)i * n + order[idx].first];
      if (v > 0) b[(size_t)i * n + idx] = v;
    }
  std::copy(b.begin(), b.end(), a);
  compress(a, n, out);
}

void compress_skip_order(double* a, int n, Compressed* out) {
  std::vector<int> deg(n, 0), row_perm, col_perm;
  std::vector<char> used(n, 0), visited(n, 0);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      if (a[(size_t)i * n + j] != 0) deg[j]++;
  for (int step = 0; step < n; step++) {
    int cur = -1, best = INT_MAX;
    for (int l = 0; l < n; l++)
      if (!used[l] && deg[l] < best) {
        best = deg[l];
        cur = l;
      }
    used[cur] = 1;
    col_perm.push_back(cur);
    for (int l = 0; l < n; l++) {
      if (a[(size_t)l * n + cur] != 0 && !visited[l]) {
        visited[l] = 1;
        row_perm.push_back(l);
        for (int k = 0; k < n; k++)
          if (a[(size_t)l * n + k] != 0 && !used[k]) deg[k]--;
      }
    }
  }
  for (int l = 0; l < n; l++)
    if (!visited[l]) row_perm.push_back(l);
  std::vector<double> prev(a, a + (size_t)n * n);
  for (int r = 0; r < n; r++)
    for (int c = 0; c < n; c++) a[(size_t)r * n + c] = prev[(size_t)row_perm[r] * n + col_perm[c]];
  compress(a, n, out);
}

std::string grid_graph(int m, int n, HostMatrix* out) {
  if (m < 1 || n < 1) return "grid sides must be positive";
  if ((m & 1) && (n & 1)) return "one of the grid sides must be even";
  // iterate over `rows` x `cols` cells with `cols` even
  const int rows = (m % 2 == 0) ? n : m;
  const int cols = (m % 2 == 0) ? m : n;
  const int nov = m * n / 2;
  if (nov > 4096) return "grid too large";
  out->n = nov;
  out->header_nnz = 0;
  out->type = "int";
  out->a.assign((size_t)nov * nov, 0.0);
  const int half = cols / 2;
  for (int i = 0; i < rows; i++) {
    for (int j = 0; j < cols; j++) {
      const int x = i * half + j / 2;
      int nb[4], k = 0;
      if (x - half >= 0) nb[k++] = x - half;  // cell above
      if (x + half < nov) nb[k++] = x + half;  // cell below
      if (j % 2 == 0) {  // horizontal neighbours share index x or x-1
        if (j != 0) nb[k++] = x - 1;
        nb[k++] = x;
      } else {
        nb[k++] = x;
        if (j != cols - 1) nb[k++] = x + 1;
      }
      const bool black = ((i + j) & 1) == 0;  // black cells are rows, white cells columns
      for (int t = 0; t < k; t++) {
        if (black)
          out->a[(size_t)x * nov + nb[t]] = 1.0;
        else
          out->a[(size_t)nb[t] * nov + x] = 1.0;
      }
    }
  }
  return "";
}

void compress_mode(int mode, double* a, int n, Compressed* out) {
  if (mode == 1)
    compress_sort_order(a, n, out);
  else if (mode == 2)
    compress_skip_order(a, n, out);
  else
    compress(a, n, out);
}

}  // namespace perm
