// Operator-pass instantiations for float.
#include "ops3d.cuh"

namespace omb {
template cudaError_t launch_op<float>(OpKind, const OpUnit<float>*, int, int, int, int, const TwTables&,
                                   cudaStream_t);
template cudaError_t launch_op3d<float>(OpKind, const OpUnit<float>*, int, int, int, int, int, const TwTables&,
                                     OpUnit<float>*, cudaStream_t);
}  // namespace omb
