// pipeline_host.h - host-side interface of the fused LBVH + OBB-tree +
// collapse build (pipeline.cu) for other parts of the library.
#pragma once

#include <cstddef>
#include <cstdint>

namespace obvh {
namespace pipeline {

// Byte offsets, inside a build workspace for n triangles, of the words that
// obvh_build_status reads: the build's error word, the collapse's primitive
// slot count, and the LBVH stage's error word (all u32).
struct StatusWords {
    size_t error, slots, lbvh_error;
};
StatusWords status_words(uint32_t n);

}  // namespace pipeline
}  // namespace obvh
