// Operator-pass instantiations for double.
#include "ops3d.cuh"

namespace omb {
template cudaError_t launch_op<double>(OpKind, const OpUnit<double>*, int, int, int, int, const TwTables&,
                                   cudaStream_t);
template cudaError_t launch_op3d<double>(OpKind, const OpUnit<double>*, int, int, int, int, int, const TwTables&,
                                     OpUnit<double>*, cudaStream_t);
}  // namespace omb
