/*
 * ref_treelet_emu.cpp - TEST INFRASTRUCTURE ONLY.  Runs the reference's own
 * ATRBVH treelet kernel, agglomerativeSmallTreelet Kernel
 * (src/ads/atrbvh_gpu/AgglomerativeTreelet.cu:14-222,405-570, with formTreelet
 * from Treelet.cuh:21-129 and the index maps of TriangularMatrix.cuh:34-52),
 * as HOST code, one warp at a time, so that the treelet restatement in
 * oracle/atrbvh_oracle.c and the CUDA path can be checked against the
 * reference's code itself.  The kernel is never run on a GPU as a checker:
 * launched as shipped (128-thread blocks) its __syncthreads() sit in loops
 * whose trip counts differ between the warps of a block.
 *
 * How the kernel runs here
 *   - oracle/Makefile compiles AgglomerativeTreelet.cu from the reference tree
 *     with two textual edits that leave the algorithm alone: the
 *     `extern __shared__` array becomes a plain `extern` array (defined below,
 *     shared by the 32 lanes of the running warp), and the kernel launchers
 *     after the kernels (`<<<...>>>` syntax) are cut off.
 *   - Each lane of a warp is a fiber with its own stack (x86-64 context switch
 *     below).  Every warp intrinsic (__shfl_sync, __shfl_down_sync,
 *     __ballot_sync) and __syncthreads() is a barrier: all 32 lanes run up to
 *     it, then the exchange happens.  A round in which the lanes reach
 *     different intrinsics (divergent warp intrinsics) is an error, reported
 *     to the caller.
 *   - The kernel also relies on the warp running converged between
 *     intrinsics in two places: (1) distances written by all lanes in
 *     calculateDistancesMatrix / updateDistancesMatrix are read by all lanes
 *     at the top of the next findMinimumDistance; (2) in updateTreelet every
 *     lane tests `treeletLeavesAreas[1] < nodesSah[treeletInternalNodes[0]]`
 *     before lane 1 overwrites that node's SAH.  (1) gets a barrier at the
 *     start of findMinimumDistance (hooked through its FLT_MAX), (2) holds
 *     because the lanes of a round run from lane 31 down to lane 0.
 *   - Warps run one after another.  The kernel's bottom-up walk has no waits
 *     (the second thread to reach a node continues, the first stops), and a
 *     treelet only reads and writes the subtree of its root, which is final
 *     when its root is reached, so this is one of the schedules the GPU can
 *     run and gives the tree every schedule gives.
 *   - The warp of thread t is t / 32, as in the reference's 128-thread blocks
 *     (blockDim is 32 here, one warp per block).
 *   - The optimisation loop is AgglomerativeTreeletOptimizer::Optimize
 *     (AgglomerativeTreeletOptimizer.cpp:22-98) for treelets of at most 20
 *     leaves: counters cleared, the small-treelet kernel, gamma doubled, per
 *     iteration.  The schedule comes from the reference's own
 *     AgglomerativeScheduler::GenerateScheduleLower.
 * Arithmetic is compiled without contraction (-ffp-contract=off), like the
 * other host checkers here.
 */
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <device_launch_parameters.h>
#include <vector_types.h>

#include "AgglomerativeScheduler.h"
#include "AgglomerativeTreelet.h"
#include "BVHTree.h"
#include "Commons.cuh"
#include "TimeKernelExecution.h"
#include "TriangularMatrix.cuh"

// ------------------------------------------------------------------ fibers
extern "C" void obvh_emu_switch(void** save_sp, void* load_sp);
__asm__(
    ".text\n"
    ".p2align 4\n"
    ".globl obvh_emu_switch\n"
    ".hidden obvh_emu_switch\n"
    ".type obvh_emu_switch,@function\n"
    "obvh_emu_switch:\n"
    "  pushq %rbp\n"
    "  pushq %rbx\n"
    "  pushq %r12\n"
    "  pushq %r13\n"
    "  pushq %r14\n"
    "  pushq %r15\n"
    "  subq $16, %rsp\n"
    "  stmxcsr 8(%rsp)\n"
    "  fnstcw (%rsp)\n"
    "  movq %rsp, (%rdi)\n"
    "  movq %rsi, %rsp\n"
    "  ldmxcsr 8(%rsp)\n"
    "  fldcw (%rsp)\n"
    "  addq $16, %rsp\n"
    "  popq %r15\n"
    "  popq %r14\n"
    "  popq %r13\n"
    "  popq %r12\n"
    "  popq %rbx\n"
    "  popq %rbp\n"
    "  ret\n"
    ".size obvh_emu_switch, .-obvh_emu_switch\n");

namespace obvh_emu {

enum Op : int { kOpShfl = 1, kOpShflDown, kOpBallot, kOpSync, kOpConverge, kOpDone };

constexpr int kLanes = 32;
constexpr size_t kStackBytes = 256 * 1024;

struct Lane {
    void* sp = nullptr;
    uint64_t count = 0;  // intrinsics passed
    int op = 0;          // the intrinsic this lane waits at (kOpDone: returned)
};

Lane g_lane[kLanes];
std::vector<unsigned char> g_stacks;
void* g_main_sp = nullptr;
int g_cur = 0;
uint3 g_block_idx;
const char* g_fault = nullptr;
uint32_t g_xchg[2][kLanes];
void (*g_body)() = nullptr;

void lane_main();

// Round over: every lane must wait at the same intrinsic (or have returned).
// Returns the lane to run next, or -1 for "back to the host".
int end_of_round() {
    const int op = g_lane[0].op;
    const uint64_t count = g_lane[0].count;
    for (int l = 1; l < kLanes; ++l)
        if (g_lane[l].op != op || g_lane[l].count != count) {
            g_fault = "ref_treelet_emu: the lanes of a warp reached different warp intrinsics";
            return -1;
        }
    return op == kOpDone ? -1 : kLanes - 1;
}

// The running lane stops at an intrinsic (or has returned); run the next one.
void yield(int op) {
    const int me = g_cur;
    g_lane[me].op = op;
    if (op != kOpDone) g_lane[me].count++;
    const int next = me > 0 ? me - 1 : end_of_round();
    if (next < 0) {
        obvh_emu_switch(&g_lane[me].sp, g_main_sp);
    } else {
        g_cur = next;
        obvh_emu_switch(&g_lane[me].sp, g_lane[next].sp);
    }
    // resumed: the scheduler set g_cur to this lane again
}

void lane_main() {
    g_body();
    yield(kOpDone);
    // a returned lane is never resumed: its frame is rebuilt for the next warp
    for (;;) obvh_emu_switch(&g_lane[g_cur].sp, g_main_sp);
}

// Build lane l's first frame: obvh_emu_switch pops it and "returns" into
// lane_main with the stack aligned as after a call.
void init_lane(int l) {
    unsigned char* top = g_stacks.data() + (l + 1) * kStackBytes;
    top = reinterpret_cast<unsigned char*>(reinterpret_cast<uintptr_t>(top) & ~uintptr_t(15));
    uint64_t* sp = reinterpret_cast<uint64_t*>(top - 80);
    std::memset(sp, 0, 80);
    uint16_t fpu_cw = 0x037F;
    uint32_t mxcsr = 0x1F80;
    std::memcpy(reinterpret_cast<unsigned char*>(sp), &fpu_cw, sizeof(fpu_cw));
    std::memcpy(reinterpret_cast<unsigned char*>(sp) + 8, &mxcsr, sizeof(mxcsr));
    sp[8] = reinterpret_cast<uint64_t>(&lane_main);  // return address
    g_lane[l].sp = sp;
    g_lane[l].count = 0;
    g_lane[l].op = 0;
}

// Run `body` as one warp of 32 lanes; returns the fault message or null.
const char* run_warp(unsigned block, void (*body)()) {
    if (g_stacks.empty()) g_stacks.resize(kLanes * kStackBytes);
    g_block_idx = make_uint3(block, 0, 0);
    g_body = body;
    g_fault = nullptr;
    for (int l = 0; l < kLanes; ++l) init_lane(l);
    g_cur = kLanes - 1;
    obvh_emu_switch(&g_main_sp, g_lane[g_cur].sp);
    return g_fault;
}

__attribute__((noinline)) uint3 thread_idx() { return make_uint3(static_cast<unsigned>(g_cur), 0, 0); }
__attribute__((noinline)) uint3 block_idx() { return g_block_idx; }
inline dim3 block_dim() { return dim3(kLanes, 1, 1); }

void check_mask(unsigned mask) {
    if (mask != 0xffffffffu) g_fault = "ref_treelet_emu: partial-warp mask";
}

template <class T>
T shfl_sync(unsigned mask, T v, int src) {
    static_assert(sizeof(T) == 4, "32-bit shuffles only");
    check_mask(mask);
    const int me = g_cur, b = static_cast<int>(g_lane[me].count & 1);
    std::memcpy(&g_xchg[b][me], &v, 4);
    yield(kOpShfl);
    T r;
    std::memcpy(&r, &g_xchg[b][src & (kLanes - 1)], 4);
    return r;
}

template <class T>
T shfl_down_sync(unsigned mask, T v, unsigned delta) {
    static_assert(sizeof(T) == 4, "32-bit shuffles only");
    check_mask(mask);
    const int me = g_cur, b = static_cast<int>(g_lane[me].count & 1);
    std::memcpy(&g_xchg[b][me], &v, 4);
    yield(kOpShflDown);
    const unsigned src = static_cast<unsigned>(me) + delta;
    if (src >= static_cast<unsigned>(kLanes)) return v;  // out of range: own value
    T r;
    std::memcpy(&r, &g_xchg[b][src], 4);
    return r;
}

unsigned ballot_sync(unsigned mask, int pred) {
    check_mask(mask);
    const int me = g_cur, b = static_cast<int>(g_lane[me].count & 1);
    g_xchg[b][me] = pred ? 1u : 0u;
    yield(kOpBallot);
    unsigned r = 0;
    for (int l = 0; l < kLanes; ++l) r |= g_xchg[b][l] << l;
    return r;
}

void syncthreads() { yield(kOpSync); }

// FLT_MAX as the kernel reads it; at the top of findMinimumDistance it also
// stands for the converged warp of the GPU: every lane's distance writes land
// before any lane reads the matrix.
float flt_max_at(const char* function) {
    if (std::strcmp(function, "findMinimumDistance") == 0) yield(kOpConverge);
    return __FLT_MAX__;
}

template <class T, class U>
T atomic_add(T* address, U v) {  // lanes never run at the same time
    const T old = *address;
    *address = static_cast<T>(old + v);
    return old;
}

}  // namespace obvh_emu

// ------------------------------------------------------------------ the kernel
#undef __global__
#undef __device__
#undef __host__
#undef __forceinline__
#undef __shared__
#undef FLT_MAX
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static
#define threadIdx (::obvh_emu::thread_idx())
#define blockIdx (::obvh_emu::block_idx())
#define blockDim (::obvh_emu::block_dim())
#define __shfl_sync ::obvh_emu::shfl_sync
#define __shfl_down_sync ::obvh_emu::shfl_down_sync
#define __ballot_sync ::obvh_emu::ballot_sync
#define __syncthreads ::obvh_emu::syncthreads
#define __threadfence() ((void)0)
#define __ffs __builtin_ffs
#define atomicAdd ::obvh_emu::atomic_add
#define FLT_MAX (::obvh_emu::flt_max_at(__func__))

// the kernel's dynamic shared memory (one warp per block; 249 words at 20 leaves)
int sharedMemory[4096];

#include "treelet_kernel_host.inc"

#undef FLT_MAX
#define FLT_MAX __FLT_MAX__

// The reference's SoA tree class has a private constructor befriended to this
// class name; the reference's own manager (device copies) is not linked.
class BVHTreeInstanceManager {
public:
    static SoABVHTree* view(unsigned n, int* parent, int* left, int* right, int* data, float4* lo, float4* hi,
                            float* area) {
        SoABVHTree* t = new SoABVHTree(n, false);
        t->data.parentIndices = parent;
        t->data.leftIndices = left;
        t->data.rightIndices = right;
        t->data.dataIndices = data;
        t->data.boundingBoxMin = lo;
        t->data.boundingBoxMax = hi;
        t->data.area = area;
        t->data.rootIndex = 0;
        return t;
    }
    static void release(SoABVHTree* t) {
        t->data.parentIndices = nullptr;
        t->data.leftIndices = nullptr;
        t->data.rightIndices = nullptr;
        t->data.dataIndices = nullptr;
        t->data.boundingBoxMin = nullptr;
        t->data.boundingBoxMax = nullptr;
        t->data.area = nullptr;
        delete t;
    }
};

namespace {
struct KernelArgs {
    unsigned n;
    BVHTree* tree;
    int treelet_size;
    int* subtree_triangles;
    unsigned* counters;
    int gamma;
    const int* schedule;
    int schedule_size;
    int distance_matrix_size;
    float* nodes_sah;
    float ci, ct;
} g_args;

void small_treelet_lane() {
    const KernelArgs& a = g_args;
    agglomerativeSmallTreeletKernel(a.n, a.tree, a.treelet_size, a.subtree_triangles, a.counters, a.gamma,
                                    a.schedule, a.schedule_size, a.distance_matrix_size, a.nodes_sah, a.ci, a.ct);
}
}  // namespace

/* Optimise the SoA tree in place (n triangles, 2n-1 nodes, root 0, leaves
 * from n-1): the reference's treelet optimisation for treelets of 3..20
 * leaves.  Arrays are the reference's SoABVHTree fields.  Returns 0, or -1
 * with the reason in *error. */
extern "C" int ref_treelet_optimize(unsigned n, int treelet_size, int iterations, float ci, float ct, int* parent,
                                    int* left, int* right, int* data, float* lo4, float* hi4, float* area,
                                    const char** error) {
    *error = nullptr;
    if (n < 2 || treelet_size < 3 || treelet_size > 20 || iterations < 0) {
        *error = "ref_treelet_optimize: unsupported arguments (n >= 2, 3 <= treelet size <= 20)";
        return -1;
    }
    const size_t nodes = 2 * static_cast<size_t>(n) - 1;
    BVHTree* tree = BVHTreeInstanceManager::view(n, parent, left, right, data, reinterpret_cast<float4*>(lo4),
                                                 reinterpret_cast<float4*>(hi4), area);
    std::vector<unsigned> counters(n - 1);
    std::vector<int> subtree(nodes);
    std::vector<float> sah(nodes);
    AgglomerativeScheduler scheduler;
    std::vector<int> schedule;
    int schedule_size = 0;
    scheduler.GenerateScheduleLower(treelet_size, 32, schedule, schedule_size);
    const int matrix = sumArithmeticSequence(treelet_size - 1, 1, treelet_size - 1);

    int gamma = treelet_size;
    const unsigned warps = (n + 31) / 32;
    int rc = 0;
    for (int it = 0; it < iterations && rc == 0; ++it) {
        std::fill(counters.begin(), counters.end(), 0u);
        g_args = KernelArgs{n,          tree,      treelet_size,  subtree.data(), counters.data(), gamma,
                            schedule.data(), schedule_size, matrix, sah.data(),      ci,              ct};
        for (unsigned w = 0; w < warps; ++w) {
            if (const char* f = obvh_emu::run_warp(w, &small_treelet_lane)) {
                *error = f;
                rc = -1;
                break;
            }
        }
        gamma *= 2;
    }
    BVHTreeInstanceManager::release(tree);
    return rc;
}
