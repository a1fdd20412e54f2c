/*
 * Test harness: the host-side pointer rule of dg-rain_b200/csrc/dgr_ptr.h, compiled for the
 * host alone, so that its answers for memory a single-GPU machine cannot produce (another
 * GPU's buffer, an unmapped pinned buffer) are checked on the CPU.  Not part of the library.
 */
#include "../dg-rain_b200/csrc/dgr_ptr.h"

extern "C" int dgr_t_may_access(int type, int owner_device, const void *device_pointer, const void *p, int device)
{
    return dgr_kernel_may_access(type, owner_device, device_pointer, p, device) ? 1 : 0;
}

extern "C" int dgr_t_memory_types(int *out)
{
    out[0] = cudaMemoryTypeUnregistered;
    out[1] = cudaMemoryTypeHost;
    out[2] = cudaMemoryTypeDevice;
    out[3] = cudaMemoryTypeManaged;
    return 4;
}
