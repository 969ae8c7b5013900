// prog_wind.cu -- the wind at particle positions, interpolated from the resident flow field
// (Zeitschleife.IntWindCalculate, Intwind.cs:31-152): the consumer of the solved field in GRAL's
// Lagrangian particle tracking.  One thread per particle; the field reads are gathers of two
// neighbouring values per component, the level search runs over HOKART in shared memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "prog_ctx.cuh"

namespace gral {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxLevels = 4096;   // HOKART entries staged in shared memory (NKK + 2)

struct WindArgs {
    int nii, njj, nkk;
    float dxk, dyk, ahmin;
    int ikooa, jkooa, terrain, buildings;
    const float *uk, *vk, *wk;      // one situation's fields, flat [NII+2][NJJ+2][NKK+2]
    const float *hok, *dzk;         // [NKK+2]
    int nh;                         // flat terrain without buildings: met profile
    const float *mh, *ou, *ov;      // [nh+1]
    float expo;                     // exponent of the power law (from Ob[1][1], on the host)
};

// BinarySearch of Intwind.cs:162-197: first level whose HOKART is at or above h, starting from
// the split at NKK/8, capped at NKK
__device__ __forceinline__ int level_search(const float *hok, int nkk, float h) {
    int low = 1, high = nkk;
    const int eighth = high >> 3;
    if (hok[eighth] >= h) high = eighth;
    else low = eighth;
    while (low <= high) {
        const int mid = (low + high) >> 1;
        if (hok[mid] >= h) high = mid - 1;
        else low = mid + 1;
    }
    return (low > nkk) ? nkk : low;
}

// u1 + (u2 - u1) / D * (x - (origin + (I - 1) * D)): the cell origin is int + float in float, the
// offset from the double particle coordinate and the product in double (Intwind.cs:47-53)
__device__ __forceinline__ float lerp_face(float a, float b, float d, double x, int origin, int idx) {
    const float base = (float)origin + (float)(idx - 1) * d;
    const float slope = (b - a) / d;
    return (float)((double)a + (double)slope * (x - (double)base));
}

__global__ void __launch_bounds__(kThreads) k_wind_at(WindArgs a, int n, const gral_particle *__restrict__ p,
                                                      float *__restrict__ ux, float *__restrict__ uy,
                                                      float *__restrict__ uz, int *__restrict__ kidx, int *bad) {
    extern __shared__ float s_hok[];
    for (int k = threadIdx.x; k < a.nkk + 2; k += blockDim.x) s_hok[k] = a.hok[k];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const gral_particle q = p[t];
    float UX = 0.f, UY = 0.f, UZ = 0.f;
    int K = 0;
    const bool field = a.terrain || a.buildings;
    if (field && (q.i < 1 || q.i > a.nii || q.j < 1 || q.j > a.njj)) {
        *bad = 1;
        ux[t] = uy[t] = uz[t] = __int_as_float(0x7fc00000);
        kidx[t] = 0;
        return;
    }
    if (field) {
        float hz;   // height in the HOKART frame for W
        if (a.terrain) {
            const float f1 = q.z - a.ahmin;
            K = level_search(s_hok, a.nkk, f1);
            hz = f1;
        } else {
            for (K = 1; K <= a.nkk; ++K)
                if (q.z <= s_hok[K]) break;
            if (K > a.nkk) K = a.nkk;
            hz = q.z + q.ahint;
        }
        const int nj2 = a.njj + 2, nk2 = a.nkk + 2;
        const size_t c = ((size_t)q.i * nj2 + q.j) * nk2 + K;
        UX = lerp_face(a.uk[c], a.uk[c + (size_t)nj2 * nk2], a.dxk, q.x, a.ikooa, q.i);
        UY = lerp_face(a.vk[c], a.vk[c + nk2], a.dyk, q.y, a.jkooa, q.j);
        const float w1 = a.wk[c], w2 = a.wk[c + 1];
        UZ = w1 + (w2 - w1) / a.dzk[K] * (hz - s_hok[K - 1]);
    } else {
        // the met profile (Intwind.cs:66-117)
        const float z = q.z;
        if (z <= a.mh[1]) {
            const float dumfac = (float)pow((double)(z / a.mh[1]), (double)a.expo);
            UX = a.ou[1] * dumfac;
            UY = a.ov[1] * dumfac;
        } else if (z >= a.mh[a.nh]) {
            if (a.nh == 1) {
                const float dumfac = (float)pow((double)(z / a.mh[a.nh]), (double)a.expo);
                UX = a.ou[a.nh] * dumfac;
                UY = a.ov[a.nh] * dumfac;
            } else {
                UX = a.ou[a.nh];
                UY = a.ov[a.nh];
            }
        } else {
            int ipo = 1;
            for (int q2 = 1; q2 <= a.nh; ++q2)
                if (z > a.mh[q2]) ipo = q2 + 1;
            const float help = 1.0f / (a.mh[ipo] - a.mh[ipo - 1]) * (z - a.mh[ipo - 1]);
            UX = a.ou[ipo - 1] + (a.ou[ipo] - a.ou[ipo - 1]) * help;
            UY = a.ov[ipo - 1] + (a.ov[ipo] - a.ov[ipo - 1]) * help;
        }
    }
    ux[t] = UX;
    uy[t] = UY;
    uz[t] = UZ;
    kidx[t] = K;
}

// MathF.Max(float, float): IEEE 754:2019 maximum
inline float host_net_max(float a, float b) {
    if (a != b) { if (!std::isnan(a)) return (b < a) ? a : b; return a; }
    return std::signbit(b) ? a : b;
}

float (*volatile c_powf)(float, float) = ::powf;

}  // namespace

}  // namespace gral

using namespace gral;

extern "C" int gral_prog_wind_at(gral_ctx *ctx, int32_t situation, const gral_wind_grid *g, const float *dzk,
                                 const float *hokart, int32_t n, const gral_particle *particles, float *ux,
                                 float *uy, float *uz, int32_t *index_k) {
    if (!ctx) return GRAL_EINVAL;
    if (!g || (n > 0 && (!particles || !ux || !uy || !uz || !index_k)))
        return fail(ctx, GRAL_EINVAL, "null pointer");
    if (n < 0) return fail(ctx, GRAL_EINVAL, "negative particle count");
    const bool field = g->terrain || g->buildings;
    if (field && (!dzk || !hokart)) return fail(ctx, GRAL_EINVAL, "null DZK or HOKART");
    if (field && (!ctx->loaded || !ctx->stored)) return fail(ctx, GRAL_ESTATE, "wind interpolation before store");
    if (field && (situation < 0 || situation >= ctx->nb)) return fail(ctx, GRAL_EINVAL, "situation index out of range");
    const gral_met *m = g->met;
    if (!field && (!m || m->n_heights < 1 || !m->measurement_height || !m->obs_u || !m->obs_v))
        return fail(ctx, GRAL_EINVAL, "the profile branch needs the met profile");
    // the profile branch reads neither the field nor the level heights
    const int NII = field ? ctx->nii : 0, NJJ = field ? ctx->njj : 0, NKK = field ? ctx->nkk : 0;
    if (NKK + 2 > kMaxLevels) return fail(ctx, GRAL_ETOOLARGE, "more than 4094 levels");
    if (n == 0) return GRAL_OK;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    PrepBufs &b = ctx->prep;
    const int nh = field ? 0 : m->n_heights;
    CK(b.points.ensure((size_t)n * sizeof(gral_particle)));
    CK(b.fields.ensure(3 * (size_t)n));
    CK(b.ints.ensure((size_t)n + 1));
    CK(b.tab.ensure(2 * (size_t)(NKK + 2) + 3 * (size_t)(nh + 1)));
    float *d_hok = b.tab.p, *d_dzk = d_hok + (NKK + 2), *d_mh = d_dzk + (NKK + 2), *d_ou = d_mh + (nh + 1),
          *d_ov = d_ou + (nh + 1);
    if (field) {
        CK(cudaMemcpyAsync(d_hok, hokart, (NKK + 2) * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_dzk, dzk, (NKK + 2) * 4, cudaMemcpyHostToDevice, st));
    }
    float expo = 0.f;
    if (!field) {
        CK(cudaMemcpyAsync(d_mh, m->measurement_height, (nh + 1) * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_ou, m->obs_u, (nh + 1) * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_ov, m->obs_v, (nh + 1) * 4, cudaMemcpyHostToDevice, st));
        const float ob = m->ob_length;   // Program.Ob[1][1] (Intwind.cs:70-77)
        expo = (ob <= 0) ? host_net_max(0.35f - 0.4f * c_powf(std::fabs(ob), -0.15f), 0.05f)
                         : 0.56f * c_powf(ob, -0.15f);
    }
    CK(cudaMemcpyAsync(b.points.p, particles, (size_t)n * sizeof(gral_particle), cudaMemcpyHostToDevice, st));
    int *d_bad = b.ints.p + n;
    CK(cudaMemsetAsync(d_bad, 0, sizeof(int), st));
    WindArgs a{};
    a.nii = NII; a.njj = NJJ; a.nkk = NKK;
    a.dxk = g->dxk; a.dyk = g->dyk; a.ahmin = g->ahmin;
    a.ikooa = g->ikooa; a.jkooa = g->jkooa; a.terrain = g->terrain; a.buildings = g->buildings;
    if (field) {
        const size_t o = ctx->sg.stride * (size_t)situation;
        a.uk = ctx->sg.uk + o; a.vk = ctx->sg.vk + o; a.wk = ctx->sg.wk + o;
    }
    a.hok = d_hok; a.dzk = d_dzk;
    a.nh = nh; a.mh = d_mh; a.ou = d_ou; a.ov = d_ov; a.expo = expo;
    float *d_u = b.fields.p, *d_v = d_u + n, *d_w = d_v + n;
    CK(cudaEventRecord(ctx->ev[0], st));
    k_wind_at<<<(n + kThreads - 1) / kThreads, kThreads, (NKK + 2) * sizeof(float), st>>>(
        a, n, reinterpret_cast<const gral_particle *>(b.points.p), d_u, d_v, d_w, b.ints.p, d_bad);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[1], st));
    int hbad = 0;
    CK(cudaMemcpyAsync(&hbad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ux, d_u, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(uy, d_v, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(uz, d_w, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(index_k, b.ints.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->prep_ms = ms;
    if (hbad) return fail(ctx, GRAL_EINVAL, "a particle's cell lies outside 1..NII x 1..NJJ");
    return GRAL_OK;
}
