// Chain kernel variants for 4 LJ types: entries in registers (1 or 2 per worker) or
// streamed (256 or 512 threads), plain or split old pass, FP64 arithmetic.
#include "yamc_chain.cuh"

namespace yamc {

#ifdef YAMC_ONE_VARIANT  // development builds: fewer instantiations
#define YAMC_EPTS(X) X(-1) X(0) X(2)
#else
#define YAMC_EPTS(X) X(-1) X(0) X(1) X(2)
#endif

template <int EPT, bool MX>
static int launch_split(const LaunchCfg &L, bool split, cudaStream_t s, int nrep, const ChainArgs &a) {
    return split ? launch_chain_t<4, EPT, true, MX>(L, s, nrep, a) : launch_chain_t<4, EPT, false, MX>(L, s, nrep, a);
}

template <int EPT, bool MX>
static int clusters_split(const LaunchCfg &L, bool split, int *out) {
    return split ? max_clusters_t<4, EPT, true, MX>(L, out) : max_clusters_t<4, EPT, false, MX>(L, out);
}

int launch_chain_t4(const LaunchCfg &L, bool split, bool mx, cudaStream_t s, int nrep, const ChainArgs &a) {
#define YAMC_CASE(E)                                                                   \
    if (L.EPT == E) {                                                                  \
        if (mx) { if (false) return launch_split<E, false>(L, split, s, nrep, a); }         \
        else return launch_split<E, false>(L, split, s, nrep, a);                      \
    }
    YAMC_EPTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("no chain kernel variant for this launch shape and precision");
    return YAMC_ELIMITS;
}

int max_clusters_t4(const LaunchCfg &L, bool split, bool mx, int *out) {
#define YAMC_CASE(E)                                                                   \
    if (L.EPT == E) {                                                                  \
        if (mx) { if (false) return clusters_split<E, false>(L, split, out); }              \
        else return clusters_split<E, false>(L, split, out);                           \
    }
    YAMC_EPTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("no chain kernel variant for this launch shape and precision");
    return YAMC_ELIMITS;
}

}  // namespace yamc
