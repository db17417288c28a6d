/*
 * ref_dito_harness.cpp - TEST INFRASTRUCTURE ONLY.  C entry point around the
 * reference's own DiTO::DiTO_14<float> (src/common/algorithm/dito/dito.cpp,
 * compiled from the reference tree by oracle/Makefile) that applies the
 * kr_points_obb clamp of src/common/geometry.cpp:232-252.  Used to pin the
 * restatement in dito_oracle.c and as the bench's reference CPU arm.
 */
#include "common/algorithm/dito/dito.h"
#include <stdint.h>
#include <thread>
#include <vector>

extern "C" void ref_dito14(const float* xyz, int64_t n, float out[15]) {
    DiTO::OBB<float> obb;
    DiTO::DiTO_14<float>((DiTO::Vector<float>*)xyz, (int)n, obb);
    const DiTO::Vector<float>* f[5] = { &obb.mid, &obb.v0, &obb.v1, &obb.v2, &obb.ext };
    for (int k = 0; k < 5; k++) { out[3 * k] = f[k]->x; out[3 * k + 1] = f[k]->y; out[3 * k + 2] = f[k]->z; }
    for (int k = 12; k < 15; k++) out[k] = (out[k] < 0.001f) ? 0.001f : out[k];
}

/* Fits many independent point sets (CSR offsets) with up to `threads` host
 * threads, one set at a time per thread: the reference has no batched path,
 * so this is how its CPU DiTO is run over a batch. */
extern "C" void ref_dito14_batch(const float* xyz, const int64_t* offsets, int64_t sets,
                                 float* out, int threads) {
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([=]() {
            for (int64_t s = t; s < sets; s += threads)
                ref_dito14(xyz + 3 * offsets[s], offsets[s + 1] - offsets[s], out + 15 * s);
        });
    }
    for (auto& th : pool) th.join();
}
