// ryser_dense_3l_r28.cu -- FP64-X dense Ryser kernels in the three-level
// row layout whose columns 1 and 2 touch rows 0..27 only and column 0
// rows 0..R1-1 (R1 in 8, 12, 16, 20), orders 30..48.
#include "ryser_dense_2l.cuh"

namespace perm {
const void* dense_3l_kernel_r28(int n, int r1) {
  switch (n) {
    case 30:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<30, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<30, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<30, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<30, 20, 28>);
      return nullptr;
    case 31:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<31, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<31, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<31, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<31, 20, 28>);
      return nullptr;
    case 32:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<32, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<32, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<32, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<32, 20, 28>);
      return nullptr;
    case 33:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<33, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<33, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<33, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<33, 20, 28>);
      return nullptr;
    case 34:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<34, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<34, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<34, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<34, 20, 28>);
      return nullptr;
    case 35:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<35, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<35, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<35, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<35, 20, 28>);
      return nullptr;
    case 36:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<36, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<36, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<36, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<36, 20, 28>);
      return nullptr;
    case 37:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<37, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<37, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<37, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<37, 20, 28>);
      return nullptr;
    case 38:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<38, 20, 28>);
      return nullptr;
    case 39:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<39, 20, 28>);
      return nullptr;
    case 40:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<40, 20, 28>);
      return nullptr;
    case 41:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<41, 20, 28>);
      return nullptr;
    case 42:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<42, 20, 28>);
      return nullptr;
    case 43:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<43, 20, 28>);
      return nullptr;
    case 44:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<44, 20, 28>);
      return nullptr;
    case 45:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<45, 20, 28>);
      return nullptr;
    case 46:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<46, 20, 28>);
      return nullptr;
    case 47:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<47, 20, 28>);
      return nullptr;
    case 48:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 8, 28>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 12, 28>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 16, 28>);
      if (r1 == 20) return reinterpret_cast<const void*>(&ryser_dense_3l_kernel<48, 20, 28>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
