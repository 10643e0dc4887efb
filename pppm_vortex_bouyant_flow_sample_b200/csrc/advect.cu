// Advection of the vortex positions by their own velocity.
//
// pppm_advect_euler follows the reference's applyFlow for the particles
// (HFS/VortexSimulationSystemImp.cpp:277-314 calling move_particle,
// HFS/GPU_kernel.cu:3118-3140): p <- float(double(p) + u dt), w = 0.
// pppm_advect_rk2 is the midpoint method the at-scale workload asks for:
// u1 = U(x), x_mid = x + dt/2 u1, u2 = U(x_mid), x <- x + dt u2, with the
// strengths held fixed.  U is the full PPPM evaluation at the vortices
// themselves (segment mode against themselves, as computeURotation drives it).
#include "pppm_internal.cuh"

namespace pppm {
namespace {

__global__ void move_kernel(const float4 *__restrict__ base, const double *__restrict__ u, size_t stride, double dt,
                            uint32_t N, float4 *__restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float4 p = base[t];
    const double x = (double)p.x + u[t] * dt;
    const double y = (double)p.y + u[stride + t] * dt;
    const double z = (double)p.z + u[2 * stride + t] * dt;
    out[t] = make_float4((float)x, (float)y, (float)z, 0.0f);
}

}  // namespace

cudaError_t launch_move(pppm_scene *s, const float4 *base, const double *u, size_t stride, double dt, uint32_t N,
                        float4 *out) {
    ::pppm::note_launch();
    move_kernel<<<(N + 255) / 256, 256, 0, s->stream>>>(base, u, stride, dt, N, out);
    return cudaGetLastError();
}

}  // namespace pppm
