// ryser_dense_intc_sparse_g4p.cu -- certified int32-X dense Ryser kernels in the
// two-level row layout, groups of 4 rows multiplied in int64 pairs: orders 20..48, 1..3 outer groups.
#include "ryser_dense_intc_sparse.cuh"

namespace perm {
const void* dense_intc_sparse_kernel_g4p(int n, int ngo) {
  switch (n) {
    case 20:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<20, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<20, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<20, 4, true, 3>);
      return nullptr;
    case 21:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<21, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<21, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<21, 4, true, 3>);
      return nullptr;
    case 22:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<22, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<22, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<22, 4, true, 3>);
      return nullptr;
    case 23:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<23, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<23, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<23, 4, true, 3>);
      return nullptr;
    case 24:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<24, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<24, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<24, 4, true, 3>);
      return nullptr;
    case 25:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<25, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<25, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<25, 4, true, 3>);
      return nullptr;
    case 26:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<26, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<26, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<26, 4, true, 3>);
      return nullptr;
    case 27:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<27, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<27, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<27, 4, true, 3>);
      return nullptr;
    case 28:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<28, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<28, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<28, 4, true, 3>);
      return nullptr;
    case 29:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<29, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<29, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<29, 4, true, 3>);
      return nullptr;
    case 30:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<30, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<30, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<30, 4, true, 3>);
      return nullptr;
    case 31:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<31, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<31, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<31, 4, true, 3>);
      return nullptr;
    case 32:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<32, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<32, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<32, 4, true, 3>);
      return nullptr;
    case 33:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<33, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<33, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<33, 4, true, 3>);
      return nullptr;
    case 34:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<34, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<34, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<34, 4, true, 3>);
      return nullptr;
    case 35:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<35, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<35, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<35, 4, true, 3>);
      return nullptr;
    case 36:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<36, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<36, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<36, 4, true, 3>);
      return nullptr;
    case 37:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<37, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<37, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<37, 4, true, 3>);
      return nullptr;
    case 38:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<38, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<38, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<38, 4, true, 3>);
      return nullptr;
    case 39:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<39, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<39, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<39, 4, true, 3>);
      return nullptr;
    case 40:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<40, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<40, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<40, 4, true, 3>);
      return nullptr;
    case 41:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<41, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<41, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<41, 4, true, 3>);
      return nullptr;
    case 42:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<42, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<42, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<42, 4, true, 3>);
      return nullptr;
    case 43:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<43, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<43, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<43, 4, true, 3>);
      return nullptr;
    case 44:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<44, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<44, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<44, 4, true, 3>);
      return nullptr;
    case 45:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<45, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<45, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<45, 4, true, 3>);
      return nullptr;
    case 46:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<46, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<46, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<46, 4, true, 3>);
      return nullptr;
    case 47:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<47, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<47, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<47, 4, true, 3>);
      return nullptr;
    case 48:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<48, 4, true, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<48, 4, true, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_intc_sparse_kernel<48, 4, true, 3>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
