// Chain kernel variants for YAMC_NT LJ types.  build.py compiles this file once per LJ type
// count (-DYAMC_NT=1..4), so the variants compile in parallel: entries in registers (1 or 2 per
// worker) or streamed (256-thread or wide CTAs), plain or split old pass, FP64 or mixed
// arithmetic (the mixed form for up to 3 LJ types: SPC/E + Na + Cl).
#include "yamc_chain.cuh"

#ifndef YAMC_NT
#error "compile once per LJ type count with -DYAMC_NT=1..4"
#endif

namespace yamc {

#ifdef YAMC_ONE_VARIANT  // development builds: fewer instantiations
#define YAMC_EPTS(X) X(-1) X(0) X(2)
#else
#define YAMC_EPTS(X) X(-1) X(0) X(1) X(2)
#endif

namespace {
constexpr int NT = YAMC_NT;
constexpr bool kMixedBuilt = NT <= 3;

template <int EPT, bool MX>
int launch_split(const LaunchCfg &L, bool split, cudaStream_t s, int nrep, const ChainArgs &a) {
    return split ? launch_chain_t<NT, EPT, true, MX>(L, s, nrep, a) : launch_chain_t<NT, EPT, false, MX>(L, s, nrep, a);
}

template <int EPT, bool MX>
int clusters_split(const LaunchCfg &L, bool split, int *out) {
    return split ? max_clusters_t<NT, EPT, true, MX>(L, out) : max_clusters_t<NT, EPT, false, MX>(L, out);
}
}  // namespace

template <>
int launch_chain_nt<NT>(const LaunchCfg &L, bool split, bool mx, cudaStream_t s, int nrep, const ChainArgs &a) {
#define YAMC_CASE(E)                                                                        \
    if (L.EPT == E) {                                                                       \
        if (!mx) return launch_split<E, false>(L, split, s, nrep, a);                       \
        if constexpr (kMixedBuilt) return launch_split<E, kMixedBuilt>(L, split, s, nrep, a); \
    }
    YAMC_EPTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("no chain kernel variant for this launch shape and precision");
    return YAMC_ELIMITS;
}

template <>
int max_clusters_nt<NT>(const LaunchCfg &L, bool split, bool mx, int *out) {
#define YAMC_CASE(E)                                                                \
    if (L.EPT == E) {                                                               \
        if (!mx) return clusters_split<E, false>(L, split, out);                    \
        if constexpr (kMixedBuilt) return clusters_split<E, kMixedBuilt>(L, split, out); \
    }
    YAMC_EPTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("no chain kernel variant for this launch shape and precision");
    return YAMC_ELIMITS;
}

}  // namespace yamc
