// ryser_dense_inst_1.cu -- instantiations of the dense Ryser kernel for
// orders 21..32 (split across files so they compile in parallel).
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_1(int n) {
  switch (n) {
    case 21: return reinterpret_cast<const void*>(&ryser_dense_kernel<21>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_kernel<22>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_kernel<23>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_kernel<24>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_kernel<25>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_kernel<26>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_kernel<27>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_kernel<28>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_kernel<29>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_kernel<30>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_kernel<31>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_kernel<32>);
    default: return nullptr;
  }
}
}  // namespace perm
