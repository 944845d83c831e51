// ryser_dense_inst_4.cu -- instantiations of the dense Ryser kernel for
// orders 53..64 (split across files so they compile in parallel).
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_4(int n) {
  switch (n) {
    case 53: return reinterpret_cast<const void*>(&ryser_dense_kernel<53>);
    case 54: return reinterpret_cast<const void*>(&ryser_dense_kernel<54>);
    case 55: return reinterpret_cast<const void*>(&ryser_dense_kernel<55>);
    case 56: return reinterpret_cast<const void*>(&ryser_dense_kernel<56>);
    case 57: return reinterpret_cast<const void*>(&ryser_dense_kernel<57>);
    case 58: return reinterpret_cast<const void*>(&ryser_dense_kernel<58>);
    case 59: return reinterpret_cast<const void*>(&ryser_dense_kernel<59>);
    case 60: return reinterpret_cast<const void*>(&ryser_dense_kernel<60>);
    case 61: return reinterpret_cast<const void*>(&ryser_dense_kernel<61>);
    case 62: return reinterpret_cast<const void*>(&ryser_dense_kernel<62>);
    case 63: return reinterpret_cast<const void*>(&ryser_dense_kernel<63>);
    case 64: return reinterpret_cast<const void*>(&ryser_dense_kernel<64>);
    default: return nullptr;
  }
}
}  // namespace perm
