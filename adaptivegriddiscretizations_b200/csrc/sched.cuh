// Device scheduler shared by the eikonal and the adjoint solvers: per-instance
// epochs over tiles, one global queue of tiles, no grid-wide barrier.  See
// eikonal.cu for the scheduling scheme.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "agd_common.cuh"
#include "agd_internal.h"

namespace agd {

// ------------------------------------------------------------- variants ---
enum Variant {
    V_ISO2_8 = 0, V_ISO2_16, V_RIEM2_8, V_ISO3_4, V_RIEM3_4, V_RIEM2_16,
    // multiprecision
    V_ISO2_8_MP, V_ISO2_16_MP, V_RIEM2_8_MP, V_ISO3_4_MP, V_RIEM3_4_MP,
    // source factorisation
    V_ISO2_8_F, V_ISO2_16_F, V_RIEM2_8_F, V_ISO3_4_F, V_RIEM3_4_F,
    // second order scheme
    V_ISO2_8_O2, V_ISO2_16_O2, V_RIEM2_8_O2, V_ISO3_4_O2, V_RIEM3_4_O2,
    // walls (Riemann; the Riemann variants above with multiprecision, factorisation
    // or second order read the wall bits themselves; Isotropic needs none)
    V_RIEM2_8_W, V_RIEM2_16_W, V_RIEM3_4_W,
    // Diagonal: plain, multiprecision, factorisation, second order
    V_DIAG2_8, V_DIAG2_16, V_DIAG3_4, V_DIAG2_8_MP, V_DIAG2_16_MP, V_DIAG3_4_MP,
    V_DIAG2_8_F, V_DIAG2_16_F, V_DIAG3_4_F, V_DIAG2_8_O2, V_DIAG2_16_O2, V_DIAG3_4_O2,
    // Rander: plain, walls, multiprecision, factorisation, second order
    V_RAND2_8, V_RAND3_4, V_RAND2_8_W, V_RAND3_4_W, V_RAND2_8_MP, V_RAND3_4_MP, V_RAND2_8_F, V_RAND3_4_F,
    V_RAND2_8_O2, V_RAND3_4_O2,
    // source factorisation with multiprecision (the default tile shapes)
    V_ISO2_16_FMP, V_RIEM2_8_FMP, V_ISO3_4_FMP, V_RIEM3_4_FMP,
    // second order scheme with source factorisation, and with multiprecision
    V_ISO2_16_O2F, V_RIEM2_8_O2F, V_ISO3_4_O2F, V_RIEM3_4_O2F,
    V_ISO2_16_O2MP, V_RIEM2_8_O2MP, V_ISO3_4_O2MP, V_RIEM3_4_O2MP,
    // second order scheme with source factorisation and multiprecision
    V_ISO2_16_O2FMP, V_RIEM2_8_O2FMP, V_ISO3_4_O2FMP, V_RIEM3_4_O2FMP, V_COUNT
};
static_assert(V_COUNT <= 64, "variant masks are 64-bit");
constexpr unsigned long long kMpVariants = (1ull << V_ISO2_8_MP) | (1ull << V_ISO2_16_MP) | (1ull << V_RIEM2_8_MP) |
                                 (1ull << V_ISO3_4_MP) | (1ull << V_RIEM3_4_MP) | (1ull << V_DIAG2_8_MP) |
                                 (1ull << V_DIAG2_16_MP) | (1ull << V_DIAG3_4_MP) | (1ull << V_RAND2_8_MP) |
                                 (1ull << V_RAND3_4_MP) | (1ull << V_ISO2_16_FMP) | (1ull << V_RIEM2_8_FMP) |
                                 (1ull << V_ISO3_4_FMP) | (1ull << V_RIEM3_4_FMP) | (1ull << V_ISO2_16_O2MP) |
                                 (1ull << V_RIEM2_8_O2MP) | (1ull << V_ISO3_4_O2MP) | (1ull << V_RIEM3_4_O2MP) |
                                 (1ull << V_ISO2_16_O2FMP) | (1ull << V_RIEM2_8_O2FMP) | (1ull << V_ISO3_4_O2FMP) |
                                 (1ull << V_RIEM3_4_O2FMP);
constexpr unsigned long long kFactorVariants = (1ull << V_ISO2_8_F) | (1ull << V_ISO2_16_F) | (1ull << V_RIEM2_8_F) |
                                     (1ull << V_ISO3_4_F) | (1ull << V_RIEM3_4_F) | (1ull << V_DIAG2_8_F) |
                                     (1ull << V_DIAG2_16_F) | (1ull << V_DIAG3_4_F) | (1ull << V_RAND2_8_F) |
                                     (1ull << V_RAND3_4_F);
constexpr unsigned long long kOrder2Variants = (1ull << V_ISO2_8_O2) | (1ull << V_ISO2_16_O2) | (1ull << V_RIEM2_8_O2) |
                                     (1ull << V_ISO3_4_O2) | (1ull << V_RIEM3_4_O2) | (1ull << V_DIAG2_8_O2) |
                                     (1ull << V_DIAG2_16_O2) | (1ull << V_DIAG3_4_O2) | (1ull << V_RAND2_8_O2) |
                                     (1ull << V_RAND3_4_O2) | (1ull << V_ISO2_16_O2F) | (1ull << V_RIEM2_8_O2F) |
                                     (1ull << V_ISO3_4_O2F) | (1ull << V_RIEM3_4_O2F) | (1ull << V_ISO2_16_O2MP) |
                                     (1ull << V_RIEM2_8_O2MP) | (1ull << V_ISO3_4_O2MP) | (1ull << V_RIEM3_4_O2MP) |
                                     (1ull << V_ISO2_16_O2FMP) | (1ull << V_RIEM2_8_O2FMP) |
                                     (1ull << V_ISO3_4_O2FMP) | (1ull << V_RIEM3_4_O2FMP);
// second order with factorisation / with multiprecision / with both
constexpr unsigned long long kOrder2FactorVariants = (1ull << V_ISO2_16_O2F) | (1ull << V_RIEM2_8_O2F) |
                                           (1ull << V_ISO3_4_O2F) | (1ull << V_RIEM3_4_O2F);
constexpr unsigned long long kOrder2MpVariants = (1ull << V_ISO2_16_O2MP) | (1ull << V_RIEM2_8_O2MP) |
                                       (1ull << V_ISO3_4_O2MP) | (1ull << V_RIEM3_4_O2MP);
constexpr unsigned long long kOrder2FactorMpVariants = (1ull << V_ISO2_16_O2FMP) | (1ull << V_RIEM2_8_O2FMP) |
                                             (1ull << V_ISO3_4_O2FMP) | (1ull << V_RIEM3_4_O2FMP);
constexpr unsigned long long kWallVariants = (1ull << V_RIEM2_8_W) | (1ull << V_RIEM2_16_W) | (1ull << V_RIEM3_4_W) |
                                           (1ull << V_RAND2_8_W) | (1ull << V_RAND3_4_W);
constexpr unsigned long long kDiagVariants = ((1ull << (V_DIAG3_4_O2 + 1)) - 1) & ~((1ull << V_DIAG2_8) - 1);
constexpr unsigned long long kRanderVariants = ((1ull << (V_RAND3_4_O2 + 1)) - 1) & ~((1ull << V_RAND2_8) - 1);

static int base_variant_of(const agd_instance &a);

static int variant_of(const agd_instance &a) {
    const int v = base_variant_of(a);
    if (v >= 0 && a.order2_threshold > 0.f) {
        const bool mp = a.multip_step != 0.f, fact = a.factor_radius2 > 0.f;
        if (mp || fact) {  // the default tile shapes
            switch (v) {
                case V_ISO2_16: return mp && fact ? V_ISO2_16_O2FMP : mp ? V_ISO2_16_O2MP : V_ISO2_16_O2F;
                case V_RIEM2_8: return mp && fact ? V_RIEM2_8_O2FMP : mp ? V_RIEM2_8_O2MP : V_RIEM2_8_O2F;
                case V_ISO3_4: return mp && fact ? V_ISO3_4_O2FMP : mp ? V_ISO3_4_O2MP : V_ISO3_4_O2F;
                case V_RIEM3_4: return mp && fact ? V_RIEM3_4_O2FMP : mp ? V_RIEM3_4_O2MP : V_RIEM3_4_O2F;
                default: return -1;
            }
        }
        switch (v) {
            case V_ISO2_8: return V_ISO2_8_O2;
            case V_ISO2_16: return V_ISO2_16_O2;
            case V_RIEM2_8: return V_RIEM2_8_O2;
            case V_ISO3_4: return V_ISO3_4_O2;
            case V_RIEM3_4: return V_RIEM3_4_O2;
            case V_DIAG2_8: return V_DIAG2_8_O2;
            case V_DIAG2_16: return V_DIAG2_16_O2;
            case V_DIAG3_4: return V_DIAG3_4_O2;
            case V_RAND2_8: return V_RAND2_8_O2;
            case V_RAND3_4: return V_RAND3_4_O2;
            default: return -1;
        }
    }
    if (v >= 0 && a.factor_radius2 > 0.f) {
        if (a.multip_step != 0.f) {
            switch (v) {
                case V_ISO2_16: return V_ISO2_16_FMP;
                case V_RIEM2_8: return V_RIEM2_8_FMP;
                case V_ISO3_4: return V_ISO3_4_FMP;
                case V_RIEM3_4: return V_RIEM3_4_FMP;
                default: return -1;  // no build of factorisation with multiprecision for this model / tile
            }
        }
        switch (v) {
            case V_ISO2_8: return V_ISO2_8_F;
            case V_ISO2_16: return V_ISO2_16_F;
            case V_RIEM2_8: return V_RIEM2_8_F;
            case V_ISO3_4: return V_ISO3_4_F;
            case V_RIEM3_4: return V_RIEM3_4_F;
            case V_DIAG2_8: return V_DIAG2_8_F;
            case V_DIAG2_16: return V_DIAG2_16_F;
            case V_DIAG3_4: return V_DIAG3_4_F;
            case V_RAND2_8: return V_RAND2_8_F;
            case V_RAND3_4: return V_RAND3_4_F;
            default: return -1;
        }
    }
    if (v < 0) return v;
    if (a.multip_step == 0.f) {
        if (a.wall_dist && (a.model == AGD_MODEL_RIEMANN || a.model == AGD_MODEL_RANDER)) {
            switch (v) {
                case V_RIEM2_8: return V_RIEM2_8_W;
                case V_RIEM2_16: return V_RIEM2_16_W;
                case V_RIEM3_4: return V_RIEM3_4_W;
                case V_RAND2_8: return V_RAND2_8_W;
                case V_RAND3_4: return V_RAND3_4_W;
                default: return -1;
            }
        }
        return v;
    }
    switch (v) {
        case V_ISO2_8: return V_ISO2_8_MP;
        case V_ISO2_16: return V_ISO2_16_MP;
        case V_RIEM2_8: return V_RIEM2_8_MP;
        case V_ISO3_4: return V_ISO3_4_MP;
        case V_RIEM3_4: return V_RIEM3_4_MP;
        case V_DIAG2_8: return V_DIAG2_8_MP;
        case V_DIAG2_16: return V_DIAG2_16_MP;
        case V_DIAG3_4: return V_DIAG3_4_MP;
        case V_RAND2_8: return V_RAND2_8_MP;
        case V_RAND3_4: return V_RAND3_4_MP;
        default: return -1;  // no multiprecision build of this tile shape
    }
}

// The variant without multiprecision.
static int base_variant_of(const agd_instance &a) {
    if (a.ndim == 2) {
        if (a.model == AGD_MODEL_RIEMANN && a.shape_i[0] == 8 && a.shape_i[1] == 8) return V_RIEM2_8;
        if (a.model == AGD_MODEL_RIEMANN && a.shape_i[0] == 16 && a.shape_i[1] == 16) return V_RIEM2_16;
        if (a.model == AGD_MODEL_ISOTROPIC && a.shape_i[0] == 8 && a.shape_i[1] == 8) return V_ISO2_8;
        if (a.model == AGD_MODEL_ISOTROPIC && a.shape_i[0] == 16 && a.shape_i[1] == 16) return V_ISO2_16;
        if (a.model == AGD_MODEL_DIAGONAL && a.shape_i[0] == 8 && a.shape_i[1] == 8) return V_DIAG2_8;
        if (a.model == AGD_MODEL_DIAGONAL && a.shape_i[0] == 16 && a.shape_i[1] == 16) return V_DIAG2_16;
        if (a.model == AGD_MODEL_RANDER && a.shape_i[0] == 8 && a.shape_i[1] == 8) return V_RAND2_8;
    } else if (a.ndim == 3 && a.shape_i[0] == 4 && a.shape_i[1] == 4 && a.shape_i[2] == 4) {
        if (a.model == AGD_MODEL_RIEMANN) return V_RIEM3_4;
        if (a.model == AGD_MODEL_ISOTROPIC) return V_ISO3_4;
        if (a.model == AGD_MODEL_DIAGONAL) return V_DIAG3_4;
        if (a.model == AGD_MODEL_RANDER) return V_RAND3_4;
    }
    return -1;
}

// Epoch lists per instance: two (by epoch parity), or kMaxLists in a plan whose
// instances have release epochs (a tile pushed before its release epoch waits
// in the list of that epoch, at most kMaxLists - 1 epochs ahead).
constexpr int kMaxLists = 32;

// Per-instance epoch state.
struct InstState {
    int epoch;         // current epoch (1-based)
    int pending;       // tiles of the current epoch not yet finished
    unsigned cnt[kMaxLists];  // lengths of the instance's lists, by epoch modulo the list count
    int done;
    unsigned first;    // ticket of the first entry of epoch 1
    int changed;       // global iteration: last epoch in which a tile changed
};

struct Ctrl {
    unsigned head, tail;       // global queue tickets (monotonic)
    int active;                // instances not finished
    unsigned err;
};

// Workspace: [Inst][InstState][tile_inst][lists][flags][score0][score1][queue][Ctrl][stats]
struct WsLayout {
    size_t inst, istate, tile_inst, lists, flags, bits, score0, score1, queue, ctrl, stats, stencil, total;
    int total_tiles;
    int nlists;  // epoch lists per instance (2, or kMaxLists with release epochs)
    unsigned qcap;
};

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr long long kMaxWarps = 148 * 64;  // resident warps of a launch, upper bound
// Launches of this many instances take queue tickets in pairs (Riemann2 512^2:
// -7 % at 32 instances, +3 % at 64, +10 % at 128, +13 % at 256).
constexpr int kPairInstances = 64;

static bool layout(const agd_instance *a, int n, WsLayout &L, Inst *out, bool stencil_cache = true) {
    long long tiles = 0, stencil_floats = 0;
    bool gated = false;
    for (int i = 0; i < n; ++i) {
        gated = gated || a[i].release != nullptr;
        Inst I;
        std::memset(&I, 0, sizeof(I));
        I.a = a[i];
        if (a[i].ndim < 2 || a[i].ndim > 3) return false;
        I.size_o = 1;
        for (int k = 0; k < a[i].ndim; ++k) {
            if (a[i].shape[k] <= 0 || a[i].shape_i[k] <= 0) return false;
            I.shape_o[k] = (a[i].shape[k] + a[i].shape_i[k] - 1) / a[i].shape_i[k];
            I.size_o *= I.shape_o[k];
        }
        I.size_i = 1;
        for (int k = 0; k < a[i].ndim; ++k) I.size_i *= a[i].shape_i[k];
        I.size_tot = (long long)I.size_o * I.size_i;
        I.tile_base = (int)tiles;
        I.variant = variant_of(a[i]);
        I.stencil = nullptr;
        I.stencil_off = -1;
        if (stencil_cache && (a[i].model == AGD_MODEL_RIEMANN || a[i].model == AGD_MODEL_RANDER)) {
            I.stencil_off = stencil_floats;  // the pointer is set once the workspace is known
            stencil_floats += 2ll * (a[i].ndim * (a[i].ndim + 1) / 2) * I.size_tot;
        }
        tiles += I.size_o;
        if (tiles > 0x3fffffff) return false;
        if (out) out[i] = I;
    }
    // Queue slots: at most `tiles` entries are outstanding (an instance's current
    // epoch list), plus the tickets held by waiting warps (up to 4 a warp) and
    // the exit sentinels (as many).
    const unsigned qcap = (unsigned)(2 * tiles + 10 * kMaxWarps) | 1u;  // odd: see kSlotEmpty
    size_t off = 0;
    L.inst = off; off = align256(off + sizeof(Inst) * n);
    L.istate = off; off = align256(off + sizeof(InstState) * n);
    L.tile_inst = off; off = align256(off + sizeof(int) * tiles);
    L.nlists = gated ? kMaxLists : 2;
    L.lists = off; off = align256(off + sizeof(int) * tiles * L.nlists);
    L.flags = off; off = align256(off + sizeof(unsigned) * tiles);
    L.bits = off; off = align256(off + sizeof(unsigned) * 3 * ((tiles + 31) / 32));
    L.score0 = off; off = align256(off + sizeof(unsigned) * tiles);
    L.score1 = off; off = align256(off + sizeof(unsigned) * tiles);
    L.queue = off; off = align256(off + sizeof(unsigned long long) * qcap);
    L.ctrl = off; off = align256(off + sizeof(Ctrl));
    L.stats = off; off = align256(off + sizeof(agd_stats) * n);
    L.stencil = off; off = align256(off + sizeof(float) * stencil_floats);
    L.total = off;
    L.total_tiles = (int)tiles;
    L.qcap = qcap;
    return true;
}

static bool layout(const agd_instance *a, int n, WsLayout &L, std::vector<Inst> *out, bool stencil_cache = true) {
    if (out) out->resize(n);
    return layout(a, n, L, out ? out->data() : static_cast<Inst *>(nullptr), stencil_cache);
}

// Points the stencils of the instances at their offsets, recorded by layout(),
// in the workspace's stencil region.
static void rebase_stencils(Inst *insts, int n, const WsLayout &L, void *ws) {
    for (int i = 0; i < n; ++i)
        insts[i].stencil = insts[i].stencil_off < 0
                               ? nullptr
                               : reinterpret_cast<float *>(static_cast<char *>(ws) + L.stencil +
                                                           (size_t)insts[i].stencil_off * sizeof(float));
}

// --------------------------------------------------------- kernel context ---
struct Sched {
    const Inst *inst;
    InstState *ist;
    const int *tile_inst;
    int *lists;       // list k of instance i: lists + k * ntiles + tile_base(i)
    unsigned lmask;   // list count - 1
    int ntiles;       // tiles of the launch
    unsigned *flags, *score0, *score1;
    unsigned long long *queue;
    unsigned qcap;
    Ctrl *ctrl;
    agd_stats *stats;
    int ninst;
    int nwarps;  // worker warps of the launch
    int tgroup;  // queue tickets a warp takes per atomic on the head counter (1 or 2)
    unsigned long long timeout_ns;
    // Bitmap pushes (launches of many instances without release epochs, whose
    // epochs close_epoch_bitmap publishes): the tiles pushed for epoch r are
    // the bits of bitmap r % 3 (tile t: bit t & 31 of word t >> 5), nwords
    // words each.
    unsigned *bits;
    unsigned nwords;
    int bitmap;
};

// Queue slot encoding: ticket (low 20 bits) << 44 | epoch << 30 | tile, empty =
// all ones.  A consumer holding ticket h takes slot h % qcap only when it carries
// the low bits of h.  The only other entry a slot can hold is the previous lap's
// (ticket h - qcap): qcap is odd, so its low ticket bits differ.
constexpr unsigned long long kSlotEmpty = ~0ull;
constexpr unsigned kExitTile = 0x3fffffffu;
constexpr int kMaxEpochs = 16000;
__device__ __forceinline__ unsigned long long slot_word(unsigned ticket, int epoch, unsigned tile) {
    return ((unsigned long long)(ticket & 0xfffffu) << 44) | ((unsigned long long)(epoch & 0x3fff) << 30) |
           (tile & 0x3fffffffu);
}

__device__ __forceinline__ int ld_acquire_s32(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Relaxed (strong, unordered) forms for the queue slots.  Everything a visit
// reads that other warps write during the solve is read through L2 (ld.cg) at
// addresses that depend on the slot's tile, and the producer's release store
// of the entry makes those writes visible at L2 first; an acquire here would
// add a fence and drop the L1 copies of the read-only data (instance
// descriptors, stencils, right-hand sides) at every visit.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ int *list_of(const Sched &S, const Inst &I, int epoch) {
    return S.lists + (size_t)((unsigned)epoch & S.lmask) * S.ntiles + I.tile_base;
}

// Tile t is to be visited at epoch e+1 of its instance (pushed during epoch e),
// or, with release epochs, at its release epoch if that is later (at most
// lmask epochs ahead).  The epoch a tile is pushed for never decreases, so the
// epoch-stamped flag keeps one entry per tile and epoch.
// BITMAP false: a visitor that never runs with bitmap pushes (its code stays
// out of the visit).
template <bool BITMAP = true>
__device__ __forceinline__ void push_tile(const Sched &S, const Inst &I, int ii, int t, int e) {
    if (BITMAP && S.bitmap) {  // a bit per tile and epoch: repeated pushes merge, and nothing waits for the result
        atomicOr(S.bits + (size_t)((unsigned)(e + 1) % 3u) * S.nwords + (t >> 5), 1u << (t & 31));
        return;
    }
    int r = e + 1;
    if (S.lmask > 1u && I.a.release) r = max(r, min((int)__ldg(I.a.release + (t - I.tile_base)), e + (int)S.lmask));
    const unsigned tag = (unsigned)r;
    if (atomicMax(&S.flags[t], tag) < tag) {
        const unsigned idx = atomicAdd(&S.ist[ii].cnt[tag & S.lmask], 1u);
        list_of(S, I, r)[idx] = t;
    }
}

__device__ __forceinline__ unsigned score_at(const Sched &S, int t, int e) {
    // Score written at epoch e (0 if the tile was not visited at epoch e).
    const unsigned *arr = (e & 1) ? S.score1 : S.score0;
    const unsigned w = __ldcg(arr + t);
    return (int)(w >> 8) == e ? (w & 0xffu) : 0u;
}

// Writes the entry of `ticket` once its slot is free.  The caller has made its
// earlier writes visible (a release fence), so the entry is a relaxed store.
__device__ __forceinline__ bool put_slot(const Sched &S, unsigned ticket, int epoch, unsigned tile) {
    unsigned long long *slot = S.queue + ticket % S.qcap;
    const unsigned long long t0 = globaltimer();
    while (ld_relaxed_u64(slot) != kSlotEmpty) {  // the previous lap's entry is not yet taken
        if (globaltimer() - t0 > S.timeout_ns) {
            atomicOr(&S.ctrl->err, (unsigned)AGD_STATUS_WATCHDOG);
            return false;
        }
        __nanosleep(64);
    }
    st_relaxed_u64(slot, slot_word(ticket, epoch, tile));
    return true;
}

// Appends the n tile ids src[0..n), to be visited at epoch e, to the global queue;
// warp-cooperative.  BULK: each lane handles kPubBatch entries at a time, their
// list reads and slot checks issued together (one L2 round trip for 32 x
// kPubBatch entries instead of one per 32), at the cost of the registers that
// hold them; a slot still holding its previous lap's entry is waited for by
// put_slot.
constexpr int kPubBatch = 8;
template <bool BULK>
static __device__ void enqueue_warp(const Sched &S, const int *src, int n, int e, int lane) {
    unsigned start = 0;
    if (lane == 0) start = atomicAdd(&S.ctrl->tail, (unsigned)n);
    start = __shfl_sync(kFull, start, 0);
    fence_acq_rel();  // release: the instance state and the tiles' values before the entries
    if constexpr (BULK) {
        bool ok = true;
        for (int k0 = 0; k0 < n && ok; k0 += 32 * kPubBatch) {
            int tile[kPubBatch];
            unsigned long long prev[kPubBatch];
#pragma unroll
            for (int u = 0; u < kPubBatch; ++u) {
                const int k = k0 + 32 * u + lane;
                if (k < n) {
                    tile[u] = __ldcg(src + k);
                    prev[u] = ld_relaxed_u64(S.queue + (start + (unsigned)k) % S.qcap);
                }
            }
#pragma unroll
            for (int u = 0; u < kPubBatch; ++u) {
                const int k = k0 + 32 * u + lane;
                if (k >= n || !ok) continue;
                const unsigned ticket = start + (unsigned)k;
                if (prev[u] == kSlotEmpty) st_relaxed_u64(S.queue + ticket % S.qcap, slot_word(ticket, e, (unsigned)tile[u]));
                else ok = put_slot(S, ticket, e, (unsigned)tile[u]);
            }
        }
    } else {
        for (int k = lane; k < n; k += 32)
            if (!put_slot(S, start + (unsigned)k, e, (unsigned)__ldcg(src + k))) break;
    }
    __syncwarp();
}

// End of epoch e of instance ii (called by the warp that finished its last
// tile): publish the next list, or retire the instance.  The stop test is the
// reference's: no tile left to update, or nitermax_o epochs run
// (_solvers.py:94-120 with _StopCriterion.py:62-84, _solvers.py:53-57).
template <bool BULK>
static __device__ void close_epoch(const Sched &S, int ii, int e, int lane) {
    const Inst &I = S.inst[ii];
    InstState &st = S.ist[ii];
    // The next epoch that has tiles: e+1, or with release epochs the first of
    // e+1 .. e+lmask whose list is not empty (the epochs between are empty).
    int n = 0, en = e + 1;
    if (S.lmask > 1u) {
        const unsigned c = lane < (int)S.lmask ? atomicAdd(&st.cnt[(unsigned)(e + 1 + lane) & S.lmask], 0u) : 0u;
        const unsigned nz = __ballot_sync(kFull, c != 0u);
        if (nz) {
            const int k = __ffs(nz) - 1;
            n = (int)__shfl_sync(kFull, c, k);
            en = e + 1 + k;
        }
    } else {
        if (lane == 0) n = (int)atomicAdd(&st.cnt[(e + 1) & 1], 0u);
        n = __shfl_sync(kFull, n, 0);
    }
    // global iteration: the list holds every tile; an epoch without change ends the solve
    if ((I.a.flags & AGD_FLAG_SOLVER_GLOBAL) && atomicAdd(&st.changed, 0) < e) n = 0;
    if (n == 0 || e >= I.a.nitermax_o) {
        int last = 0;
        if (lane == 0) {
            S.stats[ii].niter_o = e;
            if (e >= I.a.nitermax_o) atomicOr(&S.stats[ii].status, (int)AGD_STATUS_NOT_CONVERGED);
            st.done = 1;
            __threadfence();
            last = atomicSub(&S.ctrl->active, 1) == 1;
        }
        last = __shfl_sync(kFull, last, 0);
        if (last) {  // every instance is done: one exit sentinel per ticket a worker warp may hold
            const int nexit = 2 * S.tgroup * S.nwarps;
            unsigned start = 0;
            if (lane == 0) start = atomicAdd(&S.ctrl->tail, (unsigned)nexit);
            start = __shfl_sync(kFull, start, 0);
            fence_acq_rel();
            for (int k = lane; k < nexit; k += 32)
                if (!put_slot(S, start + (unsigned)k, 0, kExitTile)) break;
        }
        return;
    }
    if (lane == 0) {
        st.cnt[(unsigned)e & S.lmask] = 0u;  // the list of epoch e is consumed; it is refilled for a later epoch
        st.pending = n;
        st.epoch = en;
        S.stats[ii].tile_visits += n;  // tile visits = the lengths of the published lists
        __threadfence();
    }
    __syncwarp();
    enqueue_warp<BULK>(S, list_of(S, I, en), n, en, lane);
}


// close_epoch of a bitmap launch: the tiles of epoch e + 1 are the set bits of
// bitmap (e + 1) % 3 in the instance's range, compacted in tile order into its
// list of epoch e + 1 (a warp prefix sum over the words) and published from
// there.  Bitmap (e + 2) % 3, last read when epoch e - 1 closed, is cleared for
// the pushes of epoch e + 1 before the entries go out; bitmap (e + 1) % 3 is
// only read here, and cleared when epoch e + 2 closes.
template <bool BULK>
static __device__ void close_epoch_bitmap(const Sched &S, int ii, int e, int lane) {
    const Inst &I = S.inst[ii];
    InstState &st = S.ist[ii];
    const int t0 = I.tile_base, t1 = I.tile_base + I.size_o;
    const int w0 = t0 >> 5, w1 = (t1 - 1) >> 5;
    const unsigned *B = S.bits + (size_t)((unsigned)(e + 1) % 3u) * S.nwords;
    int *list = list_of(S, I, e + 1);
    int n = 0;
    for (int wb = w0; wb <= w1; wb += 32) {
        const int w = wb + lane;
        unsigned v = 0;
        if (w <= w1) {
            v = __ldcg(B + w);
            if (w == w0) v &= ~0u << (t0 & 31);
            if (w == (t1 >> 5)) v &= (1u << (t1 & 31)) - 1u;
        }
        const int c = __popc(v);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        int k = n + incl - c;
        while (v) {
            const int b = __ffs(v) - 1;
            v &= v - 1u;
            list[k++] = (w << 5) + b;  // the tile id
        }
        n += __shfl_sync(kFull, incl, 31);
    }
    if ((I.a.flags & AGD_FLAG_SOLVER_GLOBAL) && atomicAdd(&st.changed, 0) < e) n = 0;
    if (n == 0 || e >= I.a.nitermax_o) {
        int last = 0;
        if (lane == 0) {
            S.stats[ii].niter_o = e;
            if (e >= I.a.nitermax_o) atomicOr(&S.stats[ii].status, (int)AGD_STATUS_NOT_CONVERGED);
            st.done = 1;
            __threadfence();
            last = atomicSub(&S.ctrl->active, 1) == 1;
        }
        last = __shfl_sync(kFull, last, 0);
        if (last) {
            const int nexit = 2 * S.tgroup * S.nwarps;
            unsigned start = 0;
            if (lane == 0) start = atomicAdd(&S.ctrl->tail, (unsigned)nexit);
            start = __shfl_sync(kFull, start, 0);
            fence_acq_rel();
            for (int k = lane; k < nexit; k += 32)
                if (!put_slot(S, start + (unsigned)k, 0, kExitTile)) break;
        }
        return;
    }
    unsigned *C = S.bits + (size_t)((unsigned)(e + 2) % 3u) * S.nwords;
    for (int w = w0 + lane; w <= w1; w += 32) {
        unsigned keep = 0u;  // bits of the neighbouring instances in a shared word
        if (w == w0) keep |= (1u << (t0 & 31)) - 1u;
        if (w == (t1 >> 5)) keep |= ~0u << (t1 & 31);
        if (keep) atomicAnd(C + w, keep);
        else C[w] = 0u;
    }
    if (lane == 0) {
        st.pending = n;
        st.epoch = e + 1;
        S.stats[ii].tile_visits += n;
        __threadfence();
    }
    __syncwarp();
    enqueue_warp<BULK>(S, list, n, e + 1, lane);
}

// Issues (lane 0) the copy of the 16 bytes that hold the queue slot of ticket h
// into buf (shared, 16-byte aligned) without waiting for it: take_slot reads
// it after the visit in between, so that the slot's L2 round trip overlaps the
// visit.  The queue starts 256-byte aligned and its region is padded to a
// multiple of 256 bytes, so the pair of the last slot stays in the workspace.
__device__ __forceinline__ void prefetch_slot(const Sched &S, unsigned h, unsigned long long *buf) {
    const unsigned long long *pair = S.queue + ((h % S.qcap) & ~1u);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n\tcp.async.commit_group;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(buf)), "l"(pair)
                 : "memory");
}

// Waits (lane 0) for the entry of ticket h; pre: the pair of slots copied by
// prefetch_slot for h, or NULL.  Gives up with a watchdog error if the queue
// receives no entry anywhere (no epoch of any instance ends) for timeout_ns,
// or if an error is raised.
__device__ __forceinline__ unsigned long long take_slot(const Sched &S, unsigned h, const unsigned long long *pre) {
    const unsigned idx = h % S.qcap;
    unsigned long long *slot = S.queue + idx;
    if (pre) {  // the entry was there when the copy read it: no round trip now
        asm volatile("cp.async.wait_all;" ::: "memory");
        const unsigned long long v = pre[idx & 1u];
        if (v != kSlotEmpty && (unsigned)(v >> 44) == (h & 0xfffffu)) {
            st_relaxed_u64(slot, kSlotEmpty);
            return v;
        }
    }
    unsigned seen = ld_acquire(&S.ctrl->tail);
    unsigned long long t0 = globaltimer();
    unsigned backoff = 32;
    for (unsigned it = 0;; ++it) {
        const unsigned long long v = ld_relaxed_u64(slot);
        if (v != kSlotEmpty && (unsigned)(v >> 44) == (h & 0xfffffu)) {
            st_relaxed_u64(slot, kSlotEmpty);  // the slot is free for the next lap
            return v;
        }
        if ((it & 15u) == 15u) {
            if (ld_acquire(&S.ctrl->err)) return kExitTile;
            const unsigned p = ld_acquire(&S.ctrl->tail);
            const unsigned long long now = globaltimer();
            if (p != seen) {
                seen = p;
                t0 = now;
            } else if (now - t0 > S.timeout_ns) {
                atomicOr(&S.ctrl->err, (unsigned)AGD_STATUS_WATCHDOG);
                return kExitTile;
            }
        }
        __nanosleep(backoff);
        backoff = min(backoff * 2u, 1024u);
    }
}

// Worker warps: take a tile from the queue, visit it at its instance's
// current epoch, and close the epoch when it was the last tile of it.
// Visitor provides: Args (by value), Smem (per warp), and
//   static void visit(const Sched&, const Args&, int t, int ii, int e, int lane, Smem&).
// Visitor::kMinCtas: resident 4-warp CTAs per SM that its register budget must allow.
// Visitor::kBulkPublish: publish epochs with enqueue_warp<true> (more registers
// in the worker loop, for visitors whose budget has them).
// Visitor::kBatchScheduling: the worker may run launches of many instances with
// the queue-slot prefetch, the ticket group taken ahead and bitmap pushes; a
// visitor without it keeps the worker loop of one ticket ahead and list
// pushes, and their registers (the linear visitor's budget has none to spare).
constexpr int kSmemInst = 1024;  // instances whose tile bases a CTA keeps in shared memory

// Decrement with release semantics (publishes this warp's writes); the warp
// that brings the count to zero then fences, which makes everyone else's
// writes visible to it (the acquire half is needed only there).
__device__ __forceinline__ int atomic_dec_release(int *p) {
    int old;
    asm volatile("atom.release.gpu.global.add.s32 %0, [%1], -1;" : "=r"(old) : "l"(p) : "memory");
    return old;
}

template <class Visitor, int WPB>
__global__ void __launch_bounds__(WPB * 32, Visitor::kMinCtas * 4 / WPB) sched_worker(Sched S, typename Visitor::Args VA) {
    __shared__ typename Visitor::Smem smem[WPB];
    __shared__ int s_base[kSmemInst];  // tile bases, to find a tile's instance without a global load
    __shared__ __align__(16) unsigned long long s_pre[WPB][2];  // prefetched queue slots
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool inst_in_smem = S.ninst <= kSmemInst;
    if (inst_in_smem)
        for (int i = threadIdx.x; i < S.ninst; i += blockDim.x) s_base[i] = S.inst[i].tile_base;
    __syncthreads();
    if (ld_acquire_s32(&S.ctrl->active) == 0) return;  // nothing to solve
    // Each warp holds one queue ticket ahead: the ticket for its next tile is
    // taken when a visit starts, so the atomic's latency overlaps the visit.
    // With tgroup 2 a warp takes two consecutive tickets per atomic: the head
    // counter is a single address that every visit of the launch hits, and at
    // ~250 visits/us (a batch of 128 instances) its atomics are a bound.  A
    // warp then visits two tiles of the queue in turn, which lengthens the
    // tail of a small epoch: one instance alone solves 11 % slower that way,
    // so launches of fewer than kPairInstances instances take one.  Those of
    // kPairInstances or more also hold the group after (its atomic issued a
    // group ahead), so that the ticket of the next tile is known when a visit
    // starts and the copy of its queue slot (prefetch_slot) overlaps the
    // visit; a warp then holds up to 2 tgroup tickets (the exit sentinels of
    // close_epoch cover them).  Few instances keep one ticket ahead: a tile
    // held behind a busy warp lengthens their small epochs.
    const bool ahead = Visitor::kBatchScheduling && S.tgroup > 1;
    unsigned ticket = 0, group = 0;
    int spare = 0;  // tickets of the group still ahead of `ticket`
    if (lane == 0) {
        ticket = atomicAdd(&S.ctrl->head, (unsigned)S.tgroup);
        if (ahead) group = atomicAdd(&S.ctrl->head, (unsigned)S.tgroup);  // the next group
        spare = S.tgroup - 1;
    }
    bool prefetched = false;
    while (true) {
        unsigned long long v = 0;
        if (lane == 0) v = take_slot(S, ticket, prefetched ? s_pre[warp] : nullptr);
        v = __shfl_sync(kFull, v, 0);
        const unsigned t = (unsigned)(v & 0x3fffffffull);
        const int e = (int)((v >> 30) & 0x3fff);
        if (t == kExitTile) break;  // (take_slot has waited for this warp's copies)
        if (lane == 0) {
            if (spare > 0) {
                ticket += 1u;
                --spare;
            } else if (ahead) {
                ticket = group;  // its atomic was issued a group ago
                spare = S.tgroup - 1;
                group = atomicAdd(&S.ctrl->head, (unsigned)S.tgroup);
            } else {
                ticket = atomicAdd(&S.ctrl->head, (unsigned)S.tgroup);
                spare = S.tgroup - 1;
            }
            if (ahead) prefetch_slot(S, ticket, s_pre[warp]);
        }
        prefetched = ahead;
        int ii;
        if (inst_in_smem) {
            int lo = 0, hi = S.ninst - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_base[mid] <= (int)t) lo = mid; else hi = mid - 1;
            }
            ii = lo;
        } else {
            ii = __ldg(S.tile_inst + t);
        }
        Visitor::visit(S, VA, (int)t, ii, e, lane, smem[warp]);
        int lastone = 0;
        __syncwarp();
        if (lane == 0) lastone = atomic_dec_release(&S.ist[ii].pending) == 1;
        lastone = __shfl_sync(kFull, lastone, 0);
        if (lastone) {
            fence_acq_rel();
            if (Visitor::kBatchScheduling && S.bitmap) close_epoch_bitmap<Visitor::kBulkPublish>(S, ii, e, lane);
            else close_epoch<Visitor::kBulkPublish>(S, ii, e, lane);
        }
    }
}

// ---------------------------------------------------------------- setup ---
// tile -> instance map and epoch-1 lists: tiles flagged by `trigger`, by
// ACTIVATE_ALL, or holding a seed point inside the domain (the reference's
// trigger = seedTags, _SetArgs.py:122 and _solvers.py:98-100).
// One thread per tile.  The seed bits of a tile are size_i / 32 consecutive
// words; padding bits are set, so a tile that reaches past the grid tests its
// points one by one, the others OR their words.
static __global__ void setup_tiles(Sched S, int total_tiles) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total_tiles) return;
    int lo = 0, hi = S.ninst - 1;  // bisection over the tile bases
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (S.inst[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const Inst &I = S.inst[lo];
    if (t >= I.tile_base + I.size_o) return;  // past the last tile
    const int n_o = t - I.tile_base;
    const_cast<int *>(S.tile_inst)[t] = lo;
    bool active = (I.a.flags & (AGD_FLAG_ACTIVATE_ALL | AGD_FLAG_SOLVER_GLOBAL)) != 0;
    if (I.a.trigger) {
        active = active || I.a.trigger[n_o] != 0;
    } else if (!active) {
        int xo[3] = {0, 0, 0}, r = n_o;
        bool padded = false;
        for (int k = I.a.ndim - 1; k >= 0; --k) {
            xo[k] = r % I.shape_o[k];
            r /= I.shape_o[k];
            padded = padded || (xo[k] + 1) * I.a.shape_i[k] > I.a.shape[k];
        }
        const unsigned *bits = reinterpret_cast<const unsigned *>(I.a.seedbits) + (size_t)n_o * (I.size_i >> 5);
        if (!padded) {
            unsigned any = 0;
            for (int j = 0; j < (I.size_i >> 5); ++j) any |= __ldg(bits + j);
            active = any != 0;
        } else {
            for (int n_i = 0; n_i < I.size_i && !active; ++n_i) {
                int q = n_i;
                bool in = true;
                for (int k = I.a.ndim - 1; k >= 0; --k) {
                    in = in && xo[k] * I.a.shape_i[k] + q % I.a.shape_i[k] < I.a.shape[k];
                    q /= I.a.shape_i[k];
                }
                active = in && ((__ldg(bits + (n_i >> 5)) >> (n_i & 31)) & 1u);
            }
        }
    }
    if (active) {
        S.flags[t] = 1u;
        const unsigned idx = atomicAdd(&S.ist[lo].cnt[1], 1u);
        list_of(S, I, 1)[idx] = t;
    }
}

// Epoch 1 of every instance: one warp per instance publishes its first list.
static __global__ void publish_first(Sched S) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= S.ninst) return;
    InstState &st = S.ist[ii];
    const int n = (int)st.cnt[1];
    if (n == 0) {
        st.done = 1;
        S.stats[ii].niter_o = 0;
        return;
    }
    st.cnt[0] = 0u;
    st.pending = n;
    st.epoch = 1;
    S.stats[ii].tile_visits = n;
    atomicAdd(&S.ctrl->active, 1);
    st.first = atomicAdd(&S.ctrl->tail, (unsigned)n);  // the instance's tickets for epoch 1
}

// The entries of epoch 1, one thread per tile position: the queue was just
// cleared, so every slot is free, and the workers start after this kernel.
static __global__ void publish_first_slots(Sched S, int total_tiles) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= total_tiles) return;
    int lo = 0, hi = S.ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (S.inst[mid].tile_base <= j) lo = mid; else hi = mid - 1;
    }
    const InstState &st = S.ist[lo];
    const int k = j - S.inst[lo].tile_base;
    if (k >= (int)st.cnt[1]) return;
    const unsigned ticket = st.first + (unsigned)k;
    S.queue[ticket % S.qcap] = slot_word(ticket, 1, (unsigned)list_of(S, S.inst[lo], 1)[k]);
}

static __global__ void finish_stats(Sched S, agd_stats *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ninst) return;
    agd_stats st = S.stats[i];
    st.status |= (int)S.ctrl->err;
    if (!S.ist[i].done) st.status |= (int)AGD_STATUS_WATCHDOG;
    if (out) out[i] = st;
}

// --------------------------------------------------------------- launch ---
template <class Visitor, int WPB>
static int launch_workers(const Sched &S, const typename Visitor::Args &VA, int total_tiles, const agd_launch *cfg,
                          cudaStream_t st) {
    auto kern = sched_worker<Visitor, WPB>;
    int dev = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_cuda_error("cudaGetDevice");
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WPB * 32, 0) != cudaSuccess)
        return set_cuda_error("occupancy query");
    if (per_sm < 1) return set_error(AGD_STATUS_UNSUPPORTED, "worker kernel does not fit on an SM");
    const int max_ctas = per_sm * nsm;  // all resident: idle warps wait on their queue ticket
    int ctas = cfg && cfg->ctas > 0 ? cfg->ctas : (total_tiles + WPB - 1) / WPB;
    ctas = std::max(1, std::min(ctas, max_ctas));
    Sched s = S;
    s.nwarps = ctas * WPB;
    s.tgroup = S.ninst >= kPairInstances ? 2 : 1;  // exit sentinels: 2 tgroup nwarps <= 4 kMaxWarps
    if (s.nwarps > kMaxWarps) return set_error(AGD_STATUS_INVALID, "too many worker warps");
    kern<<<ctas, WPB * 32, 0, st>>>(s, VA);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return set_cuda_error("worker launch", err);
    return AGD_STATUS_OK;
}

// Scheduler pointers inside a workspace laid out by layout().
static Sched sched_at(const WsLayout &L, void *ws, int ninst) {
    char *w = static_cast<char *>(ws);
    Sched S;
    S.inst = reinterpret_cast<const Inst *>(w + L.inst);
    S.ist = reinterpret_cast<InstState *>(w + L.istate);
    S.tile_inst = reinterpret_cast<const int *>(w + L.tile_inst);
    S.lists = reinterpret_cast<int *>(w + L.lists);
    S.lmask = (unsigned)L.nlists - 1u;
    S.ntiles = L.total_tiles;
    S.flags = reinterpret_cast<unsigned *>(w + L.flags);
    S.bits = reinterpret_cast<unsigned *>(w + L.bits);
    S.nwords = (unsigned)((L.total_tiles + 31) / 32);
    S.bitmap = 0;
    S.score0 = reinterpret_cast<unsigned *>(w + L.score0);
    S.score1 = reinterpret_cast<unsigned *>(w + L.score1);
    S.queue = reinterpret_cast<unsigned long long *>(w + L.queue);
    S.qcap = L.qcap;
    S.ctrl = reinterpret_cast<Ctrl *>(w + L.ctrl);
    S.stats = reinterpret_cast<agd_stats *>(w + L.stats);
    S.ninst = ninst;
    S.nwarps = 0;
    S.tgroup = 1;
    S.timeout_ns = 2000000000ull;
    return S;
}

// One scheduled solve over the instances already uploaded at L.inst: clears the
// scheduler state, builds the first lists, runs the workers, writes the stats.
template <class Visitor>
static int run_sched(const WsLayout &L, void *ws, int n, const typename Visitor::Args &VA, agd_stats *stats,
                     const agd_launch *cfg, cudaStream_t st) {
    Sched S = sched_at(L, ws, n);
    if (cfg && cfg->timeout_ns > 0) S.timeout_ns = (unsigned long long)cfg->timeout_ns;
    // Bitmap pushes for launches of many instances: the pushes of a visit then
    // wait for nothing, and an epoch is published in tile order.  A single
    // instance keeps the lists, whose push order (the front's) propagates
    // faster within an epoch when nothing else fills the GPU.
    S.bitmap = (Visitor::kBatchScheduling && !Visitor::kBulkPublish && L.nlists == 2 && n >= kPairInstances) ? 1 : 0;
    char *w = static_cast<char *>(ws);
    cudaError_t err = cudaMemsetAsync(w + L.istate, 0, sizeof(InstState) * n, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(w + L.flags, 0, L.queue - L.flags, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(w + L.queue, 0xff, L.ctrl - L.queue, st);
    // control block and stats; the stencil region after them is written in full by the stencil pass
    if (err == cudaSuccess) err = cudaMemsetAsync(w + L.ctrl, 0, L.stencil - L.ctrl, st);
    if (err != cudaSuccess) return set_cuda_error("workspace clear", err);
    if ((err = Visitor::prepare(S, L, st)) != cudaSuccess) return set_cuda_error("prepare", err);
    setup_tiles<<<(L.total_tiles + 255) / 256, 256, 0, st>>>(S, L.total_tiles);
    if ((err = cudaGetLastError()) != cudaSuccess) return set_cuda_error("setup_tiles", err);
    publish_first<<<(n + 127) / 128, 128, 0, st>>>(S);
    publish_first_slots<<<(L.total_tiles + 255) / 256, 256, 0, st>>>(S, L.total_tiles);
    if ((err = cudaGetLastError()) != cudaSuccess) return set_cuda_error("publish_first", err);
    // 8-warp CTAs only where their static shared memory fits in 48 KB
    constexpr bool kWide = (sizeof(typename Visitor::Smem) + 16) * 8 + sizeof(int) * kSmemInst <= 48 * 1024;
    const int rc = (kWide && cfg && cfg->warps_per_cta == 8)
                       ? launch_workers<Visitor, kWide ? 8 : 4>(S, VA, L.total_tiles, cfg, st)
                       : launch_workers<Visitor, 4>(S, VA, L.total_tiles, cfg, st);
    if (rc != AGD_STATUS_OK) return rc;
    if ((err = Visitor::finalize(S, L, st)) != cudaSuccess) return set_cuda_error("finalize", err);
    finish_stats<<<(n + 127) / 128, 128, 0, st>>>(S, stats);
    if ((err = cudaGetLastError()) != cudaSuccess) return set_cuda_error("finish_stats", err);
    return AGD_STATUS_OK;
}

}  // namespace agd
