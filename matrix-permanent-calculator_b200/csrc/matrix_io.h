// matrix_io.h -- host-side matrix input and compression for the permanent
// engine: the reference's text format and its CRS/CCS builders, restated.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace perm {

// A dense n x n matrix held row-major in double (int and float inputs are
// converted exactly; float values are first rounded to float, as the
// reference stores them in a float matrix).
struct HostMatrix {
  int n = 0;
  int header_nnz = 0;
  std::string type;  // "int" | "float" | "double"
  std::vector<double> a;
};

// Reads the reference text format (main.cu:476-488, util.h:344-358):
//   line 1: "n nnz type"   (type is int, float or double)
//   then:   "i j value"    0-based; lines that do not parse are skipped;
//   binary (the -b flag): every parsed entry is stored as 1.
// Differences from the reference, all on inputs where it has undefined
// behaviour: the matrix starts zeroed, and an index outside [0, n) is an
// error instead of an out-of-bounds write.  Returns "" or an error message.
std::string read_matrix_file(const std::string& path, bool binary, HostMatrix* out);

// CRS + CCS of the strictly positive entries (util.h:523-551: the reference
// keeps `mat > 0` only, so non-positive entries vanish from sparse paths).
struct Compressed {
  int n = 0;
  std::vector<int> cptrs, rows, rptrs, cols;
  std::vector<double> cvals, rvals;
  int nnz() const { return n ? rptrs[n] : 0; }
};
void compress(const double* a, int n, Compressed* out);

// sortOrder (util.h:554-619): columns reordered by ascending positive-entry
// count, stable among equal counts (the order glibc's merge sort gives the
// reference's comparator); `a` is rewritten in the new column order with
// non-positive entries dropped, as the reference does.
void compress_sort_order(double* a, int n, Compressed* out);

// skipOrder (util.h:622-684): greedy column order by minimum remaining degree
// (degree counts entries != 0), rows in first-touch order, `a` permuted in
// place, then compress().  Rows with no entry at all (left undefined by the
// reference) are appended in ascending order.
void compress_skip_order(double* a, int n, Compressed* out);

// Dispatch on the reference's -r value: 0 plain, 1 sortOrder, 2 skipOrder.
void compress_mode(int mode, double* a, int n, Compressed* out);

// Grid-graph input mode (util.h:403-520): the 0/1 bipartite adjacency
// between the two colour classes of an m x n board, order nov = m*n/2, whose
// permanent counts the board's domino tilings.  Cells are numbered
// row-by-row, half a row per index along the even side.  Returns "" or an
// error (both sides odd).
std::string grid_graph(int m, int n, HostMatrix* out);

}  // namespace perm
