/* Force-included when building the reference's fake-CUDA CPU shim: its
 * g1_cuda_step / g1_cuda_reset_done signatures name cudaStream_t and
 * uint8_t, which its fake_cuda.h never declares (reference
 * src/g1_kernel.cu:154,165; model/fake_cuda.h). */
#include <cstdint>
typedef void* cudaStream_t;
