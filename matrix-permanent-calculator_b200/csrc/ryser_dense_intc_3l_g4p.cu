// ryser_dense_intc_3l_g4p.cu -- certified int32-X dense Ryser kernels in the
// three-level row layout, groups of 4 rows multiplied in int64 pairs: orders 28..48 (3 CTAs per SM up to order
// 40, 2 above), 2..4 groups on the first level, 1..2 on the second.
#include "ryser_dense_intc_sparse.cuh"

namespace perm {
const void* dense_intc_3l_kernel_g4p(int n, int ng1, int ng2) {
  switch (n) {
    case 28:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<28, 4, true, 4, 2, 3>);
      return nullptr;
    case 29:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<29, 4, true, 4, 2, 3>);
      return nullptr;
    case 30:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<30, 4, true, 4, 2, 3>);
      return nullptr;
    case 31:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<31, 4, true, 4, 2, 3>);
      return nullptr;
    case 32:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<32, 4, true, 4, 2, 3>);
      return nullptr;
    case 33:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<33, 4, true, 4, 2, 3>);
      return nullptr;
    case 34:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<34, 4, true, 4, 2, 3>);
      return nullptr;
    case 35:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<35, 4, true, 4, 2, 3>);
      return nullptr;
    case 36:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<36, 4, true, 4, 2, 3>);
      return nullptr;
    case 37:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<37, 4, true, 4, 2, 3>);
      return nullptr;
    case 38:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<38, 4, true, 4, 2, 3>);
      return nullptr;
    case 39:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<39, 4, true, 4, 2, 3>);
      return nullptr;
    case 40:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 2, 1, 3>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 2, 2, 3>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 3, 1, 3>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 3, 2, 3>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 4, 1, 3>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<40, 4, true, 4, 2, 3>);
      return nullptr;
    case 41:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<41, 4, true, 4, 2, 2>);
      return nullptr;
    case 42:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<42, 4, true, 4, 2, 2>);
      return nullptr;
    case 43:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<43, 4, true, 4, 2, 2>);
      return nullptr;
    case 44:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<44, 4, true, 4, 2, 2>);
      return nullptr;
    case 45:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<45, 4, true, 4, 2, 2>);
      return nullptr;
    case 46:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<46, 4, true, 4, 2, 2>);
      return nullptr;
    case 47:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<47, 4, true, 4, 2, 2>);
      return nullptr;
    case 48:
      if (ng1 == 2 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 2, 1, 2>);
      if (ng1 == 2 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 2, 2, 2>);
      if (ng1 == 3 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 3, 1, 2>);
      if (ng1 == 3 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 3, 2, 2>);
      if (ng1 == 4 && ng2 == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 4, 1, 2>);
      if (ng1 == 4 && ng2 == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_3l_kernel<48, 4, true, 4, 2, 2>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
