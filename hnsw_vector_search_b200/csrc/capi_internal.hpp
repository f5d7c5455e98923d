#pragma once

// What the C ABI's translation units share: the handle types behind include/vdx_b200.h and the
// calling thread's last-error message (read by vdx_last_error).

#include <string>

#include "vdx/brute_force.hpp"
#include "vdx/hnsw.hpp"

struct vdx_index {
    vdx::HnswIndex index;
};
struct vdx_bruteforce {
    vdx::BruteForceIndex index;
};

namespace vdx::capi {
void set_last_error(const std::string& message);
}  // namespace vdx::capi
