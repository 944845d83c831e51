// ryser_dense_inst_3.cu -- instantiations of the dense Ryser kernel for
// orders 43..52 (split across files so they compile in parallel).
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_3(int n) {
  switch (n) {
    case 43: return reinterpret_cast<const void*>(&ryser_dense_kernel<43>);
    case 44: return reinterpret_cast<const void*>(&ryser_dense_kernel<44>);
    case 45: return reinterpret_cast<const void*>(&ryser_dense_kernel<45>);
    case 46: return reinterpret_cast<const void*>(&ryser_dense_kernel<46>);
    case 47: return reinterpret_cast<const void*>(&ryser_dense_kernel<47>);
    case 48: return reinterpret_cast<const void*>(&ryser_dense_kernel<48>);
    case 49: return reinterpret_cast<const void*>(&ryser_dense_kernel<49>);
    case 50: return reinterpret_cast<const void*>(&ryser_dense_kernel<50>);
    case 51: return reinterpret_cast<const void*>(&ryser_dense_kernel<51>);
    case 52: return reinterpret_cast<const void*>(&ryser_dense_kernel<52>);
    default: return nullptr;
  }
}
}  // namespace perm
