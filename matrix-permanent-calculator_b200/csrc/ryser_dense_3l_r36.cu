// ryser_dense_3l_r36.cu -- FP64-X dense Ryser kernels in the three-level
// row layout whose columns 1 and 2 touch rows 0..35 only and column 0
// rows 0..R1-1 (R1 in 8, 12, 16, 20), orders 38..48.
#include "ryser_dense_2l.cuh"

namespace perm {
const void* dense_3l_kernel_r36(int n, int r1) {
  switch (n) {
    case 38:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 20, 36>);
      return nullptr;
    case 39:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 20, 36>);
      return nullptr;
    case 40:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 20, 36>);
      return nullptr;
    case 41:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 20, 36>);
      return nullptr;
    case 42:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 20, 36>);
      return nullptr;
    case 43:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 20, 36>);
      return nullptr;
    case 44:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 20, 36>);
      return nullptr;
    case 45:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 20, 36>);
      return nullptr;
    case 46:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 20, 36>);
      return nullptr;
    case 47:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 20, 36>);
      return nullptr;
    case 48:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 8, 36>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 12, 36>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 16, 36>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 20, 36>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
