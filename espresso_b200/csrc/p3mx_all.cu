// Single translation unit of libp3mx.so: the kernels live in headers
// (templates plus a few plain kernels), so everything is compiled once here.
#include "engine.cu"
#include "api.cu"
#include "batch.cu"
#include "noalloc.cu"
#include "dp3m.cu"
