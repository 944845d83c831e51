// ryser_dense_2l_inst_0.cu -- FP64-X dense Ryser kernels in the two-level row
// layout with 16 or 20 inner rows, orders up to 48.
#include "ryser_dense_2l.cuh"

namespace perm {
#define PERM_2L_CASE(n, r) \
  case n: return reinterpret_cast<const void*>(&ryser_dense_2l_kernel<n, r>);
const void* dense_2l_kernel_r16(int n) {
  switch (n) {
    PERM_2L_CASE(20, 16) PERM_2L_CASE(21, 16) PERM_2L_CASE(22, 16) PERM_2L_CASE(23, 16)
    PERM_2L_CASE(24, 16) PERM_2L_CASE(25, 16) PERM_2L_CASE(26, 16) PERM_2L_CASE(27, 16)
    PERM_2L_CASE(28, 16) PERM_2L_CASE(29, 16) PERM_2L_CASE(30, 16) PERM_2L_CASE(31, 16)
    PERM_2L_CASE(32, 16) PERM_2L_CASE(33, 16) PERM_2L_CASE(34, 16) PERM_2L_CASE(35, 16)
    PERM_2L_CASE(36, 16) PERM_2L_CASE(37, 16) PERM_2L_CASE(38, 16) PERM_2L_CASE(39, 16)
    PERM_2L_CASE(40, 16) PERM_2L_CASE(41, 16) PERM_2L_CASE(42, 16) PERM_2L_CASE(43, 16)
    PERM_2L_CASE(44, 16) PERM_2L_CASE(45, 16) PERM_2L_CASE(46, 16) PERM_2L_CASE(47, 16)
    PERM_2L_CASE(48, 16)
    default: return nullptr;
  }
}
const void* dense_2l_kernel_r20(int n) {
  switch (n) {
    PERM_2L_CASE(24, 20) PERM_2L_CASE(25, 20) PERM_2L_CASE(26, 20) PERM_2L_CASE(27, 20)
    PERM_2L_CASE(28, 20) PERM_2L_CASE(29, 20) PERM_2L_CASE(30, 20) PERM_2L_CASE(31, 20)
    PERM_2L_CASE(32, 20) PERM_2L_CASE(33, 20) PERM_2L_CASE(34, 20) PERM_2L_CASE(35, 20)
    PERM_2L_CASE(36, 20) PERM_2L_CASE(37, 20) PERM_2L_CASE(38, 20) PERM_2L_CASE(39, 20)
    PERM_2L_CASE(40, 20) PERM_2L_CASE(41, 20) PERM_2L_CASE(42, 20) PERM_2L_CASE(43, 20)
    PERM_2L_CASE(44, 20) PERM_2L_CASE(45, 20) PERM_2L_CASE(46, 20) PERM_2L_CASE(47, 20)
    PERM_2L_CASE(48, 20)
    default: return nullptr;
  }
}
#undef PERM_2L_CASE
}  // namespace perm
