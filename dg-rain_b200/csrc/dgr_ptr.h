/*
 * Host-side check that a caller's pointer can be handed to a kernel on a given device.
 *
 * Entry points that take device buffers from the caller (rather than copying host arrays
 * into memory the library owns) check each pointer with cudaPointerGetAttributes before
 * launching anything, so that a wrong pointer becomes DGR_ERR_INVALID instead of a device
 * fault.  The check runs on the host only and enqueues nothing, so it is also safe inside
 * a stream capture.
 */
#pragma once

#include <cuda_runtime_api.h>

/* The rule, on the values cudaPointerGetAttributes reports for pointer p:
 *   device memory   only on its own device (a buffer of another GPU is refused: with peer
 *                   access off a kernel would fault on it, and the library never enables
 *                   peer access), and only at the address the kernel would use;
 *   managed memory  where it is mapped at p;
 *   pinned host     where it is mapped at p (unified addressing);
 *   anything else   (pageable host memory, unknown pointers) refused. */
inline bool dgr_kernel_may_access(int type, int owner_device, const void *device_pointer, const void *p, int device)
{
    switch (type) {
    case cudaMemoryTypeDevice: return owner_device == device && device_pointer == p;
    case cudaMemoryTypeManaged:
    case cudaMemoryTypeHost: return device_pointer == p;
    default: return false;
    }
}

/* The same rule applied to a live pointer; false also when the runtime cannot describe it
 * (the error it raised is cleared). */
inline bool dgr_device_addressable(const void *p, int device)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return dgr_kernel_may_access((int)a.type, a.device, a.devicePointer, p, device);
}
