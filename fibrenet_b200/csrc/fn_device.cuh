/*
 * fn_device.cuh -- small device helpers shared by the step kernels
 * (fn_kernels.cu) and the adjoint kernels (fn_adjoint.cu).
 */
#ifndef FIBRENET_DEVICE_CUH
#define FIBRENET_DEVICE_CUH

#include <cuda_runtime.h>

#include "fn_types.h"

namespace fn {

/* pos.w packs the radius (float bits, low word) and the type (high word) */
__device__ __forceinline__ float w_radius(double w) { return __int_as_float(__double2loint(w)); }
__device__ __forceinline__ int w_type(double w) { return __double2hiint(w); }

/* GETADRESS, kernel.cl:9 */
__device__ __forceinline__ int getadress(int t1, int t2, int size) {
    return (t1 < t2) ? ((size * t1) + t2 - ((t1 * (t1 + 1)) / 2))
                     : ((size * t2) + t1 - ((t2 * (t2 + 1)) / 2));
}

/* Minimum image on the axes of mask (kernel.cl:598-627, 844-870). */
__device__ __forceinline__ double min_image(const FnNet& N, double& rx, double& ry, double& rz,
                                            double length, int mask) {
    const double maxDim = N.half_box_sq;
    if (length > maxDim) {
        if ((mask & 1) && rx * rx > maxDim) rx = rx > 0.0 ? rx - N.box[0] : rx + N.box[0];
        if ((mask & 2) && ry * ry > maxDim) ry = ry > 0.0 ? ry - N.box[1] : ry + N.box[1];
        if ((mask & 4) && rz * rz > maxDim) rz = rz > 0.0 ? rz - N.box[2] : rz + N.box[2];
        length = rx * rx + ry * ry + rz * rz;
    }
    return length;
}

}  // namespace fn

#endif
