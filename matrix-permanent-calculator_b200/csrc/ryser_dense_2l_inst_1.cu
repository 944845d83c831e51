// ryser_dense_2l_inst_1.cu -- FP64-X dense Ryser kernels in the two-level row
// layout with 24 or 28 inner rows, orders up to 48.
#include "ryser_dense_2l.cuh"

namespace perm {
#define PERM_2L_CASE(n, r) \
  case n: return reinterpret_cast<const void*>(&ryser_dense_2l_kernel<n, r>);
const void* dense_2l_kernel_r24(int n) {
  switch (n) {
    PERM_2L_CASE(28, 24) PERM_2L_CASE(29, 24) PERM_2L_CASE(30, 24) PERM_2L_CASE(31, 24)
    PERM_2L_CASE(32, 24) PERM_2L_CASE(33, 24) PERM_2L_CASE(34, 24) PERM_2L_CASE(35, 24)
    PERM_2L_CASE(36, 24) PERM_2L_CASE(37, 24) PERM_2L_CASE(38, 24) PERM_2L_CASE(39, 24)
    PERM_2L_CASE(40, 24) PERM_2L_CASE(41, 24) PERM_2L_CASE(42, 24) PERM_2L_CASE(43, 24)
    PERM_2L_CASE(44, 24) PERM_2L_CASE(45, 24) PERM_2L_CASE(46, 24) PERM_2L_CASE(47, 24)
    PERM_2L_CASE(48, 24)
    default: return nullptr;
  }
}
const void* dense_2l_kernel_r28(int n) {
  switch (n) {
    PERM_2L_CASE(32, 28) PERM_2L_CASE(33, 28) PERM_2L_CASE(34, 28) PERM_2L_CASE(35, 28)
    PERM_2L_CASE(36, 28) PERM_2L_CASE(37, 28) PERM_2L_CASE(38, 28) PERM_2L_CASE(39, 28)
    PERM_2L_CASE(40, 28) PERM_2L_CASE(41, 28) PERM_2L_CASE(42, 28) PERM_2L_CASE(43, 28)
    PERM_2L_CASE(44, 28) PERM_2L_CASE(45, 28) PERM_2L_CASE(46, 28) PERM_2L_CASE(47, 28)
    PERM_2L_CASE(48, 28)
    default: return nullptr;
  }
}
#undef PERM_2L_CASE
}  // namespace perm
