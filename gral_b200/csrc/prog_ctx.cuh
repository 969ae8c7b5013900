// prog_ctx.cuh -- the solver context (gral_ctx) shared by the C-ABI translation units, with
// the device-buffer helper and the error-return macros of the entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gral_prog.h"
#include "prog_common.cuh"
#include "prog_kernels.cuh"

namespace gral {

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t count) {
        if (count <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc((void **)&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// Device buffers of the set-up entry points (gral_prog_subdomains, _flat_init, _vegetation).
struct PrepBufs {
    DevBuf<float> cutk, ahk, tab, fields, veg, cov;
    DevBuf<int> ints;
    DevBuf<int16_t> kkart;
    DevBuf<uint8_t> adv, mask;
    DevBuf<unsigned char> points;
    void release() {
        cutk.release(); ahk.release(); tab.release(); fields.release(); veg.release(); cov.release();
        ints.release(); kkart.release(); adv.release(); mask.release(); points.release();
    }
};

constexpr int kCounterSlots = 64;   // wavefront launches per phase (group sets) with own counters

struct Geom {
    SweepGeom g;
    std::vector<int> ds;
};

}  // namespace gral

// gral_ctx is the opaque handle of gral_prog.h and so lives in the global namespace; the
// translation units that include this private header all work in namespace gral.
using namespace gral;

struct gral_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    int cap_nii = 0, cap_njj = 0, cap_nkk = 0, cap_kadv = 0, cap_batch = 0;
    int il_min_batch = 32;
    int forced_variant = -1;   // GRAL_PROG_BATCH_VARIANT
    int lookahead = 8;         // GRAL_PROG_LOOKAHEAD: plain-family warps per average diagonal width
    int lookahead_p = 3;       // GRAL_PROG_LOOKAHEAD_P: the same for the pressure sweep
    int variant = -1;          // chosen launch variant of the batched family (-1: not tuned yet)
    // slab family, model 1: 0 = the diagonal-claim wavefront (fused pressure..U, then V, W);
    // 1+v = strip variant v for pressure, U, V, W; 1+strip_num_variants() = pressure..U fused on
    // strips, then V, W on strip variant 0 (-1: not tuned yet)
    int pmode = -1;
    int fstrip_grid = 0;       // grid of the fused strip launch
    int forced_pmode = -1;     // GRAL_PROG_PLAIN_MODE
    int strip_grid[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // indexed by PH_*
    float ptune_ms[16] = {0};  // autotuner timings per plain mode
    std::string err = "no error";

    // current load
    bool loaded = false;
    int nii = 0, njj = 0, nkk = 0, ks = 0, nb = 0, ncols = 0, nj2 = 0, model = 1;
    bool il = false;     // interleaved layout + batched kernel family
    int ngroups = 0;
    int it_host = 1, it_max = 0, it_min = 0, cadence = 100;
    std::vector<gral_params> params;
    std::vector<gral_fields> fields;
    KArgs ka{};
    Staging sg{};
    BcLists bc{};
    Geom geo_p, geo_u, geo_v;
    bool fused = false;        // fused pressure/velcorr/average/U wavefront (slab family, model 1)
    int fused_grid = 0;
    int lookahead_f = 6;       // GRAL_PROG_LOOKAHEAD_F: fused-kernel warps per average diagonal width
    FusedGeom fgeo{};
    DevBuf<int> fseg;
    int grid_gs[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // indexed by PH_*
    cudaGraphExec_t graph = nullptr;
    float ms_upload = 0.f;
    float tune_ms[64] = {0};                  // autotuner timings per launch variant x group-set mode

    // device buffers
    DevBuf<float> slab, stage, veg, tables, ap0, rowcarry, trace;
    DevBuf<ColMeta> meta;
    DevBuf<uint32_t> cflags;
    DevBuf<ColF> colf;
    DevBuf<ColKE> colke;
    DevBuf<short2> rcw;
    // DiagnosticFlowfield after the solve (gral_params.post_diagnostic)
    bool post_diag = false;
    int diag_grid = 0;
    DevBuf<float> ddpm, dtab, ddt;
    DevBuf<int> dflags;
    DevBuf<float> varw, z0i;
    // flow-field cache payloads (gral_prog_gff_*)
    bool stored = false;                 // the staging fields hold the last store's results
    std::vector<int16_t> h_kkart;        // KKART of the load, flat [NII+2][NJJ+2]
    DevBuf<short> gff;                   // packed or uploaded payload words
    DevBuf<uint32_t> gffoff;             // terrain-format record offsets
    DevBuf<int16_t> gffkk;               // KKART of an unpack
    DevBuf<float> gffu;                  // unpacked fields, 3 x [NII+2][NJJ+2][NKK+2]
    DevBuf<char> l2flush;                // written before each timed pack launch
    PrepBufs prep;                       // set-up entry points
    // gral_prog_load_flat: initial fields built on the device during the load (else null)
    const gral_met *flat_met = nullptr;
    const gral_flat_grid *flat_grid = nullptr;
    std::vector<float> h_ref;            // per situation: the six reference-column values of the set-up
    double prep_ms = 0.0;                // device time of the last set-up call's kernels
    DevBuf<SitDev> sit;
    DevBuf<int> flags, misc, diag, bcl, counts;
    DevBuf<unsigned int> counters;
    std::vector<SitDev> h_sit;
    std::vector<int> h_act;
    // discrete adjoint (gral_prog_vjp_forward / gral_prog_vjp): checkpoints of the forward state,
    // the states kept for one checkpoint segment, cotangent fields, reverse-sweep words
    bool adj_ready = false;
    int adj_iters = 0, adj_every = 0, adj_nwe = 0, adj_nsn = 0;
    double adj_ms_forward = 0.0;
    DevBuf<float> adj_ckpt, adj_keep, adj_lam, adj_ptab, adj_stg;
    DevBuf<SitDev> adj_cksit;
    DevBuf<int> adj_ckit;
    DevBuf<unsigned int> adj_ctr;
    DevBuf<unsigned long long> adj_slot;   // stamped cotangent words of the reverse sweeps
    DevBuf<int> adj_rcr;                   // per column: whose row carry some column reads
    DevBuf<uint8_t> adj_bits;
    cudaStream_t adj_stream = nullptr;   // recomputation of the next segment beside the reverse sweeps

    ~gral_ctx() {
        if (graph) cudaGraphExecDestroy(graph);
        DevBuf<float> *fb[] = {&slab, &stage, &veg, &tables, &ap0, &rowcarry, &trace};
        for (auto *b : fb) b->release();
        meta.release(); cflags.release(); colf.release(); sit.release(); colke.release(); rcw.release();
        ddpm.release(); dtab.release(); ddt.release(); dflags.release(); fseg.release();
        varw.release(); z0i.release();
        gff.release(); gffoff.release(); gffkk.release(); gffu.release(); l2flush.release();
        prep.release();
        flags.release(); misc.release(); diag.release(); bcl.release(); counts.release();
        counters.release();
        adj_ckpt.release(); adj_keep.release(); adj_lam.release(); adj_ptab.release(); adj_stg.release();
        adj_cksit.release(); adj_ckit.release(); adj_ctr.release(); adj_slot.release(); adj_rcr.release(); adj_bits.release();
        for (auto &e : ev) if (e) cudaEventDestroy(e);
        if (adj_stream) cudaStreamDestroy(adj_stream);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace gral {

// Slab family, model 1: keep the default schedule of the sweeps (or GRAL_PROG_PLAIN_MODE) without
// trial iterations, and size its grids (prog_host.cu).
int plain_schedule_default(gral_ctx *ctx);
// the strip variant of the separate phase launches of the loaded plain mode (pmode > 0)
int strip_variant_of(const gral_ctx *ctx);
// the loaded plain mode runs pressure..U as one fused strip launch
bool fused_strips(const gral_ctx *ctx);

inline int fail(gral_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? GRAL_ENOMEM : GRAL_ECUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

#define CK_RC(call)                \
    do {                           \
        const int rc_ = (call);    \
        if (rc_ != GRAL_OK) return rc_; \
    } while (0)

}  // namespace gral
