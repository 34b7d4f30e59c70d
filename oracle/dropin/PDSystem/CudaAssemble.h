// Test infrastructure: lets the reference's own callers of its CUDA-assembly boundary compile unchanged against
// this backend (oracle/Makefile target `dropin`): their #include "PDSystem/CudaAssemble.h" lands here first.
#include "perix_cuda_compat.h"
