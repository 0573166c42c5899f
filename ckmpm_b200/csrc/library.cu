// The library's single translation unit: the engine and the allocation-free
// entry point share one set of kernel instantiations.
#include "engine.cu"
#include "noalloc.cu"
