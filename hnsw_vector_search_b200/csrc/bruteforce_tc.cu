// Tensor-core brute force: not built yet in this revision.
#include "bruteforce.cuh"

namespace vdx::dev {

std::size_t bruteforce_tc_workspace(std::uint32_t, std::uint32_t, std::uint32_t, std::uint32_t) {
    return 16;
}

cudaError_t launch_bruteforce_tc(const BruteArgs&, void*, cudaStream_t, std::uint32_t*) {
    return cudaErrorNotSupported;
}

}  // namespace vdx::dev
