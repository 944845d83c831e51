// ryser_dense_inst_2.cu -- instantiations of the dense Ryser kernel for
// orders 33..42 (split across files so they compile in parallel).
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_2(int n) {
  switch (n) {
    case 33: return reinterpret_cast<const void*>(&ryser_dense_kernel<33>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_kernel<34>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_kernel<35>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_kernel<36>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_kernel<37>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_kernel<38>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_kernel<39>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_kernel<40>);
    case 41: return reinterpret_cast<const void*>(&ryser_dense_kernel<41>);
    case 42: return reinterpret_cast<const void*>(&ryser_dense_kernel<42>);
    default: return nullptr;
  }
}
}  // namespace perm
