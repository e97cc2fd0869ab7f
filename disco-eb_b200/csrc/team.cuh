// A "team" is the group of threads that owns one k-mode: one warp on the GPU.  The same
// stepper source also compiles for a single host thread (HostTeam) so that its algebra
// can be unit-tested on a CPU against the oracle.  Loops over state entries are written
// as `for (i = T.lane; i < n; i += T.nl)`, with T.sync() between phases.
#pragma once

#include "dual.cuh"

namespace dscb {

#if defined(__CUDACC__)
struct WarpTeam {
    int lane;
    static constexpr int nl = 32;
    static constexpr int chunk = 4;         // elements per load batch in the chain substitutions
    static constexpr bool reconverge = true;  // explicit reconvergence after divergent table lookups
    static constexpr bool mixed = false;      // FP32 chain factors + FP64 refinement (ModeMem::Af)
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ double sum(double x) const
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        return x;
    }
    __device__ __forceinline__ bool leader() const { return lane == 0; }
    __device__ __forceinline__ double bcast(double x, int src) const { return __shfl_sync(0xffffffffu, x, src); }
    template <class B> __device__ __forceinline__ DualT<B> bcast(const DualT<B>& x, int src) const
    {
        return DualT<B>(bcast(x.v, src), bcast(x.d, src));
    }
    __device__ __forceinline__ bool full() const { return true; }
};
// The same warp team with element-by-element chain substitutions and no extra reconvergence
// points: measured on B200, both help a forward-solve warp (about 4 warps per SM) but slow the
// gradient block kernel (seven warps per block at the register limit), where the batched loads
// cost registers and the other warps of the block hide the divergence anyway.
struct WarpTeamSeq : WarpTeam {
    static constexpr int chunk = 1;
    static constexpr bool reconverge = false;
};
// The forward-solve warp team of the mixed-precision form (DISCOEB_METHOD_RODAS5_STRUCTURED_MIXED)
struct WarpTeamMixed : WarpTeam {
    static constexpr bool mixed = true;
};
#endif

struct HostTeam {
    int lane = 0;
    static constexpr int nl = 1;
    static constexpr int chunk = 4;
    static constexpr bool reconverge = false;
    static constexpr bool mixed = false;
    DHD void sync() const {}
    DHD double sum(double x) const { return x; }
    DHD bool leader() const { return true; }
    DHD double bcast(double x, int) const { return x; }
    template <class B> DHD DualT<B> bcast(const DualT<B>& x, int) const { return x; }
    DHD bool full() const { return false; }
};
struct HostTeamMixed : HostTeam {
    static constexpr bool mixed = true;
};

}  // namespace dscb
