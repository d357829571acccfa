// Operator-pass instantiations for double.
#include "ops_impl.cuh"

namespace omb {
template cudaError_t launch_op<double>(OpKind, const OpUnit<double>*, int, int, int, int, const TwTables&,
                                   cudaStream_t);
}  // namespace omb
