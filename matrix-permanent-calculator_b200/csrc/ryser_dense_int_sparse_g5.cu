// ryser_dense_int_sparse_g5.cu -- int32-X dense Ryser kernels in the two-level
// row layout with product groups of 5 rows: orders 20..48, 1..3 outer groups.
#include "ryser_dense_int_sparse.cuh"

namespace perm {
const void* dense_int_sparse_kernel_g5(int n, int ngo) {
  switch (n) {
    case 20:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<20, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<20, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<20, 5, 3>);
      return nullptr;
    case 21:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<21, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<21, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<21, 5, 3>);
      return nullptr;
    case 22:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<22, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<22, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<22, 5, 3>);
      return nullptr;
    case 23:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<23, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<23, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<23, 5, 3>);
      return nullptr;
    case 24:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<24, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<24, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<24, 5, 3>);
      return nullptr;
    case 25:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<25, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<25, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<25, 5, 3>);
      return nullptr;
    case 26:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<26, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<26, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<26, 5, 3>);
      return nullptr;
    case 27:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<27, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<27, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<27, 5, 3>);
      return nullptr;
    case 28:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<28, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<28, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<28, 5, 3>);
      return nullptr;
    case 29:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<29, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<29, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<29, 5, 3>);
      return nullptr;
    case 30:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<30, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<30, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<30, 5, 3>);
      return nullptr;
    case 31:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<31, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<31, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<31, 5, 3>);
      return nullptr;
    case 32:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<32, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<32, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<32, 5, 3>);
      return nullptr;
    case 33:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<33, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<33, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<33, 5, 3>);
      return nullptr;
    case 34:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<34, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<34, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<34, 5, 3>);
      return nullptr;
    case 35:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<35, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<35, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<35, 5, 3>);
      return nullptr;
    case 36:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<36, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<36, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<36, 5, 3>);
      return nullptr;
    case 37:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<37, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<37, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<37, 5, 3>);
      return nullptr;
    case 38:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<38, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<38, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<38, 5, 3>);
      return nullptr;
    case 39:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<39, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<39, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<39, 5, 3>);
      return nullptr;
    case 40:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<40, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<40, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<40, 5, 3>);
      return nullptr;
    case 41:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<41, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<41, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<41, 5, 3>);
      return nullptr;
    case 42:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<42, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<42, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<42, 5, 3>);
      return nullptr;
    case 43:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<43, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<43, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<43, 5, 3>);
      return nullptr;
    case 44:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<44, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<44, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<44, 5, 3>);
      return nullptr;
    case 45:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<45, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<45, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<45, 5, 3>);
      return nullptr;
    case 46:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<46, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<46, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<46, 5, 3>);
      return nullptr;
    case 47:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<47, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<47, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<47, 5, 3>);
      return nullptr;
    case 48:
      if (ngo == 1) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<48, 5, 1>); if (ngo == 2) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<48, 5, 2>); if (ngo == 3) return reinterpret_cast<const void*>(&ryser_dense_int_sparse_kernel<48, 5, 3>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
