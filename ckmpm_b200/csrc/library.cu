// The library's single translation unit: the engine, the allocation-free
// entry point and the differentiable rollout share one set of kernel
// instantiations.
#include "engine.cu"
#include "noalloc.cu"
#include "diff.cu"
