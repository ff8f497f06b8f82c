/* Host stand-in for cooperative_groups as used by the survivor append of shadePath
 * (src/kernels/shade_path.cu:355-363): one path per call, so the coalesced group has one
 * member and the shuffle is the identity. */
#pragma once
namespace cooperative_groups {
struct coalesced_group {
    unsigned size() const { return 1; }
    unsigned thread_rank() const { return 0; }
    template <class T> T shfl(T v, int) const { return v; }
};
inline coalesced_group coalesced_threads() { return {}; }
}
