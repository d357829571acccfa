// Operator-pass instantiations for float.
#include "ops_impl.cuh"

namespace omb {
template cudaError_t launch_op<float>(OpKind, const OpUnit<float>*, int, int, int, int, const TwTables&,
                                   cudaStream_t);
}  // namespace omb
