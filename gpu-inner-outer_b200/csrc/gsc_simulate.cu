// gsc_simulate.cu -- closed-loop simulation of a solved controller
// (gsc_problem_simulate of include/gsc_b200.h).
//
// The consumer of the controller table, plots/postprocess_controller.py of
// the reference, on the device and for many trajectories at once: one thread
// per trajectory reads the problem's device-resident controller, so nothing
// but the initial and visited states crosses PCIe.  Per sample period:
//   state_to_flat_index (:66-101)  theta wrapped with atan2(sin, cos) on a
//                                  copy, round((x - lb) / eta) (half to even)
//                                  clamped per dimension, x-fastest flat index;
//   get_control_input (:103-130)   stop at the invalid input, else the input
//                                  cell's centre (a, omega);
//   update_state (:132-176)        integration_substeps Euler substeps
//                                  x + dt * (f(x, u) + w), theta re-wrapped.
// The disturbance w is uniform in [-dhw, dhw] per dimension and substep, from
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011) keyed by the seed
// with counter (2 * (step * K + substep) + half, trajectory, 0, 0); each call
// gives two doubles ((a >> 5) * 2^26 + (b >> 6)) / 2^53, mapped as numpy's
// uniform, low + (high - low) * u.  cos, sin and atan2 are CUDA's.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gsc_internal.hpp"

using namespace gsc_api;

// Inside gsc_b200, so its exactly rounded dmul / dadd / dsub / ddiv are the
// ones found (the CUDA headers declare functions of the same names).
namespace gsc_b200 {
namespace {

struct SimArgs {
    GridInfo g;
    double dhw[4];
    const uint32_t* controller;
    const double* x0;      // [n][4]
    double* traj;          // [n][steps + 1][4] or null
    double* fin;           // [n][4] or null
    uint32_t* done;        // [n] or null
    uint32_t n;
    uint32_t steps;
    uint32_t first;        // global index of trajectory 0 of this launch (the RNG counter)
    uint32_t k0, k1;       // Philox key (the seed)
};

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// 53 random bits as a double in [0, 1): exact in every step.
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    return dmul(dadd(dmul(static_cast<double>(a >> 5), 67108864.0), static_cast<double>(b >> 6)),
                1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double wrap_atan2(double t) { return atan2(sin(t), cos(t)); }

__device__ __forceinline__ uint64_t flat_index(const GridInfo& g, const double x[4]) {
    uint64_t flat = 0, stride = 1;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const double s = d == 2 ? wrap_atan2(x[2]) : x[d];
        long long i = static_cast<long long>(rint(ddiv(dsub(s, g.lb[d]), g.eta[d])));
        if (i < 0) i = 0;
        if (i >= static_cast<long long>(g.n[d])) i = static_cast<long long>(g.n[d]) - 1;
        flat += static_cast<uint64_t>(i) * stride;
        stride *= g.n[d];
    }
    return flat;
}

__global__ void __launch_bounds__(128) k_simulate(SimArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const GridInfo& g = a.g;
    const uint32_t K = g.K;
    const double dt = g.dt;
    double x[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) x[d] = a.x0[static_cast<uint64_t>(t) * 4 + d];
    double* row = a.traj ? a.traj + static_cast<uint64_t>(t) * (a.steps + 1) * 4 : nullptr;
    if (row)
#pragma unroll
        for (int d = 0; d < 4; ++d) row[d] = x[d];
    uint32_t step = 0;
    for (; step < a.steps; ++step) {
        const uint32_t j = a.controller[flat_index(g, x)];
        if (j == kInvalid32 || j >= g.M) break;
        const double acc = input_centre(g, 0, j % g.ma);
        const double omega = input_centre(g, 1, j / g.ma);
        for (uint32_t sub = 0; sub < K; ++sub) {
            double u[4];
            for (uint32_t half = 0; half < 2; ++half) {
                uint32_t c[4] = {2u * (step * K + sub) + half, a.first + t, 0u, 0u};
                philox4x32_10(c, a.k0, a.k1);
                u[2 * half] = u53(c[0], c[1]);
                u[2 * half + 1] = u53(c[2], c[3]);
            }
            const double f[4] = {dmul(x[3], cos(x[2])), dmul(x[3], sin(x[2])), omega, acc};
            double xn[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const double low = -a.dhw[d];
                const double w = dadd(low, dmul(dsub(a.dhw[d], low), u[d]));
                xn[d] = dadd(x[d], dmul(dt, dadd(f[d], w)));
            }
            xn[2] = wrap_atan2(xn[2]);
#pragma unroll
            for (int d = 0; d < 4; ++d) x[d] = xn[d];
        }
        if (row)
#pragma unroll
            for (int d = 0; d < 4; ++d) row[static_cast<uint64_t>(step + 1) * 4 + d] = x[d];
    }
    if (row)
        for (uint32_t s = step + 1; s <= a.steps; ++s)
#pragma unroll
            for (int d = 0; d < 4; ++d) row[static_cast<uint64_t>(s) * 4 + d] = 0.0;
    if (a.fin)
#pragma unroll
        for (int d = 0; d < 4; ++d) a.fin[static_cast<uint64_t>(t) * 4 + d] = x[d];
    if (a.done) a.done[t] = step;
}

}  // namespace
}  // namespace gsc_b200

using namespace gsc_b200;

extern "C" int gsc_problem_simulate(gsc_problem* p, uint32_t count, const double* x0, uint32_t steps, uint64_t seed,
                                    double* trajectories, double* final_states, uint32_t* steps_done) {
    if (!p || (count && !x0)) return GSC_ERR_INVALID_ARGUMENT;
    gsc_context* ctx = p->ctx;
    if (!p->controller) return fail(ctx, GSC_ERR_INVALID_ARGUMENT, "problem has no controller table");
    if (static_cast<uint64_t>(steps) * p->g.K >= (1ull << 31))
        return fail(ctx, GSC_ERR_UNSUPPORTED, "steps x integration_substeps must stay below 2^31");
    if (count == 0) return GSC_OK;
    cudaGetLastError();
    GSC_CU(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    // Trajectories in chunks of at most 256 MB of device buffers.
    const uint64_t per = 4 * 8 + (trajectories ? (steps + 1ull) * 32 : 0) + (final_states ? 32 : 0) + 4;
    const uint32_t chunk = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(count, (256ull << 20) / per)));
    std::vector<std::pair<void*, uint64_t>> bufs;
    uint64_t bytes = 0;
    void* q = nullptr;
    DevicePool* pool = ctx->pool.get();
    int s = device_alloc(ctx, pool, bufs, bytes, &q, per * chunk);
    if (s != GSC_OK) return s;
    char* base = static_cast<char*>(q);
    double* dx0 = reinterpret_cast<double*>(base);
    double* dtraj = trajectories ? dx0 + 4ull * chunk : nullptr;
    double* dfin = final_states ? (dtraj ? dtraj + (steps + 1ull) * 4 * chunk : dx0 + 4ull * chunk) : nullptr;
    char* after = reinterpret_cast<char*>(dfin ? dfin + 4ull * chunk
                                               : (dtraj ? dtraj + (steps + 1ull) * 4 * chunk : dx0 + 4ull * chunk));
    uint32_t* ddone = reinterpret_cast<uint32_t*>(after);
    SimArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = p->g;
    for (int d = 0; d < 4; ++d) a.dhw[d] = p->q.dhw[d];
    a.controller = p->controller;
    a.steps = steps;
    a.k0 = static_cast<uint32_t>(seed);
    a.k1 = static_cast<uint32_t>(seed >> 32);
    cudaError_t e = cudaSuccess;
    for (uint32_t b = 0; e == cudaSuccess && b < count; b += chunk) {
        const uint32_t n = std::min(chunk, count - b);
        a.x0 = dx0;
        a.traj = dtraj;
        a.fin = dfin;
        a.done = ddone;
        a.n = n;
        a.first = b;
        e = cudaMemcpyAsync(dx0, x0 + 4ull * b, 32ull * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_simulate<<<(n + 127) / 128, 128, 0, st>>>(a);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && trajectories)
            e = cudaMemcpyAsync(trajectories + (steps + 1ull) * 4 * b, dtraj, (steps + 1ull) * 32 * n,
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && final_states)
            e = cudaMemcpyAsync(final_states + 4ull * b, dfin, 32ull * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && steps_done)
            e = cudaMemcpyAsync(steps_done + b, ddone, 4ull * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaStreamSynchronize(st);
    device_release_all(ctx, pool, bufs, bytes);
    GSC_CU(ctx, e);
    return GSC_OK;
}
