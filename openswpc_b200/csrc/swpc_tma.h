// swpc_tma.h -- launch interface of the TMA-staged 3D kernels (swpc3d_tma.cu).
#pragma once

#include <cuda_runtime.h>

#include "swpc_kernels.cuh"

namespace swpc {

// A staged launch: tiles of 32 (k) x bi (i) x bj (j) cells, and per tile the
// member groups of a batch (a single run is one member).  Field coordinates
// refer to the state slab (per member: V, S, R) and the medium slab.
struct TmaTiles {
    int nkt, nit, njt;
    int nmem, mgroups;   // members, groups of members per CTA
    int tiles_first;     // launch order: 0 member groups fastest, 1 tiles fastest
    int jblock;          // tiles of a group: k fastest, then blocks of jblock j tiles (j, then i)
    int f_v;             // state slab: Vx of member 0 (S follows at f_v + 3)
    int f_state;         // state slab: Sxx of member 0 (S, then R)
    int f_member;        // state slab: field stride between members
    int f_med;           // medium slab: lam (lam mu taup taus muyz muxz muxy)
    int f_b;             // medium slab: bx (bx by bz)
    int f_h;             // 2-byte slab of a reduced storage form: S (F16_SR) or R (BF16_R)
    long long so, ao;    // offset between members of the state arrays and of the PML auxiliaries
    int *err;            // raised when a tile copy does not complete
};

// tiles of a staged launch over a context's grid for nmem members grouped
// by mpc; nfields = the fields the kernel reads over its tile per member and
// live = the members whose tiles interleave in the launch order (both choose
// the j-block length); the field indices follow the context's slab
TmaTiles tma_tiles(const swpc_ctx *c, int bi, int bj, int nmem, int mpc, int nfields, int live);

// fields a staged stress / velocity update reads over its tile (member state
// and medium): S, R, V, lam mu taup taus muyz muxz muxy, bx by bz / V, S, bx by bz
inline int kStressFields(const swpc_ctx *c) { return 16 + 6 * c->d.nm; }
constexpr int kVelFields = 12;

// the slabs the tensor maps cover
struct TmaSlabs {
    float *state;
    long long nf_state;
    float *med;
    long long nf_med;
    void *half;           // reduced storage forms: the 2-byte fields (S for F16_SR, then R)
    long long nf_half;
};

// host copies of the tensor maps (CUtensorMap, 128 bytes, 64-byte aligned)
struct alignas(64) TmaMaps {
    unsigned char state[128];   // stress: S and R of a member (BF16_R: R; F16_SR: S and R in FP16)
    unsigned char s6[128];      // stress: S of a member (tiles without interior cells; F16_SR: FP16)
    unsigned char med[128];     // stress: the seven medium fields of the stress update
    unsigned char vh[128];      // stress: V of a member with halo
    unsigned char own3[128];    // velocity: V of a member
    unsigned char b3[128];      // velocity: bx by bz
    unsigned char va[128], vb[128], vc[128], vf[128], ve[128], vd[128];   // velocity: Sxx Syy Szz Syz Sxz Sxy
};

// compiled tiles (bi, bj) and members per CTA: stress (4,4,1) (2,4,1) (4,2,1)
// (4,2,2) (2,4,2) (2,2,2) (2,2,4) (4,1,4); velocity (4,4,1) (4,2,1) (2,2,1)
// (4,2,2) (2,2,2) (4,1,2) (2,2,4) (4,1,4).  The reduced storage forms (prec
// PREC_BF16_R / PREC_F16_SR of swpc3d_cell.cuh) run (4,4,1) and (4,2,1).
bool tma_shape_ok(int bi, int bj, int mpc, int prec = 0);
bool tma_vel_shape_ok(int bi, int bj, int mpc, int prec = 0);
bool tma_encode_stress(TmaMaps &m, const TmaSlabs &s, const Geo &g, int nm, int bi, int bj, int prec = 0);
// one FP32 map (k, i, j, field) over a slab of nf fields with box (bk, bi, bj, bf)
bool tma_encode_box(unsigned char *out, float *slab, const Geo &g, long long nf, unsigned bk, unsigned bi, unsigned bj,
                    unsigned bf);
bool tma_encode_vel(TmaMaps &m, const TmaSlabs &s, const Geo &g, int bi, int bj, int prec = 0);
cudaError_t launch_stress3d_tma(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, int bi, int bj, int mpc,
                                cudaStream_t st, int prec = 0);
cudaError_t launch_vel3d_tma(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, int bi, int bj, int mpc,
                             cudaStream_t st, int prec = 0);

}  // namespace swpc
