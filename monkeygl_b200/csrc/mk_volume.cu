// mk_volume.cu -- resident volumes: voxel texture, label texture, transfer
// function tables, per-label parameters and the brick occupancy maps used
// for empty-space skipping.
//
// Residency follows MonkeyGL's CuDataManager (core/CuDataManager.cu:28-163):
// the int16 voxels live in a 3D cudaArray (block-linear, i.e. the hardware's
// own 3D tiling) read through a normalized-coordinate, trilinear, clamped,
// normalized-float texture; labels live in a uint8 cudaArray read with
// nearest filtering at integer coordinates; each label's RGBA LUT is a 1D
// float4 array read with linear filtering.  On top of that this file keeps,
// per 8^3 brick, the voxel min/max over the brick's trilinear footprint and
// the set of labels it owns, and rebuilds a visibility bitmap whenever a
// transfer function or window changes.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "mk_internal.h"

namespace mk {

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// One warp per brick: min/max of the int16 voxels in the brick grown by one
// voxel on every side (clamped to the volume), i.e. every voxel a trilinear
// tap of an owned sample can touch.  The grown brick is at most 10x10x10;
// lanes 0-29 cover three of its 10-voxel rows at a time (lane = 10 * row +
// column) and the warp walks its rows and slices, so the loads of a warp
// are three short contiguous segments and no lane divides.  Bricks are
// numbered x fastest, so neighbouring warps share their halo rows in L2.
__global__ void __launch_bounds__(256) k_brick_minmax(const short *__restrict__ vox, int dx, int dy,
                                                      int dz, int nbx, int nby, int nbricks, short2 *out) {
    const int b = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (b >= nbricks) return;
    const int lane = threadIdx.x & 31;
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    const int x0 = max(bx * kBrick - 1, 0), x1 = min(bx * kBrick + kBrick, dx - 1);
    const int y0 = max(by * kBrick - 1, 0), y1 = min(by * kBrick + kBrick, dy - 1);
    const int z0 = max(bz * kBrick - 1, 0), z1 = min(bz * kBrick + kBrick, dz - 1);
    const int col = lane % 10, row = lane / 10;   // row 3 (lanes 30, 31) idle
    const int x = x0 + col;
    int lo = 32767, hi = -32768;
    if (row < 3 && x <= x1 && y0 + row <= y1) {
        const size_t plane = (size_t)dy * dx, step = 3 * (size_t)dx;
        const int nrows = (y1 - y0 - row) / 3 + 1;   // 3 or 4
        const short *p = vox + (size_t)z0 * plane + (size_t)(y0 + row) * dx + x;
        for (int z = z0; z <= z1; ++z, p += plane) {
            const short *q = p;
#pragma unroll 4
            for (int r = 0; r < nrows; ++r, q += step) {
                const int v = __ldg(q);
                lo = min(lo, v);
                hi = max(hi, v);
            }
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (lane == 0) out[b] = make_short2((short)lo, (short)hi);
}

// One warp per brick: the set of labels among the brick's owned voxels
// (8x8x8 at most), as a 65-bit mask in three words.  Lane = 8 * row +
// column covers four 8-byte rows at a time.
__global__ void __launch_bounds__(256) k_brick_labels(const unsigned char *__restrict__ lab, int dx,
                                                      int dy, int dz, int nbx, int nby, int nbricks,
                                                      uint32_t *out) {
    const int b = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (b >= nbricks) return;
    const int lane = threadIdx.x & 31;
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    const int x0 = bx * kBrick, x1 = min(x0 + kBrick, dx) - 1;
    const int y0 = by * kBrick, y1 = min(y0 + kBrick, dy) - 1;
    const int z0 = bz * kBrick, z1 = min(z0 + kBrick, dz) - 1;
    const int x = x0 + (lane & 7), row = lane >> 3;
    uint32_t m0 = 0, m1 = 0, m2 = 0;
    if (x <= x1 && y0 + row <= y1) {
        const size_t plane = (size_t)dy * dx, step = 4 * (size_t)dx;
        const int nrows = (y1 - y0 - row) / 4 + 1;   // 1 or 2
        const unsigned char *p = lab + (size_t)z0 * plane + (size_t)(y0 + row) * dx + x;
        for (int z = z0; z <= z1; ++z, p += plane) {
            const unsigned char *q = p;
#pragma unroll 2
            for (int r = 0; r < nrows; ++r, q += step) {
                int l = __ldg(q);
                if (l > 64) l = 64;   // labels above MAXOBJECTCOUNT never occur via the API
                if (l < 32) m0 |= 1u << l;
                else if (l < 64) m1 |= 1u << (l - 32);
                else m2 |= 1u;
            }
        }
    }
    m0 = __reduce_or_sync(0xffffffffu, m0);
    m1 = __reduce_or_sync(0xffffffffu, m1);
    m2 = __reduce_or_sync(0xffffffffu, m2);
    if (lane < 3) out[3 * (size_t)b + lane] = lane == 0 ? m0 : (lane == 1 ? m1 : m2);
}

// Label sets of the bricks of a brick-aligned sub-box (one warp per brick,
// as k_brick_labels): `lab` holds the sub-box (ex x ey x ez voxels, x
// fastest) whose first voxel is brick (bx0, by0, bz0) of the volume; the
// sets go to the volume's brick numbering and are OR-ed into present[0..2].
__global__ void __launch_bounds__(256) k_brick_labels_box(const unsigned char *__restrict__ lab, int ex, int ey,
                                                          int ez, int bx0, int by0, int bz0, int nbx, int nby,
                                                          uint32_t *out, uint32_t *present) {
    const int snbx = (ex + kBrick - 1) / kBrick, snby = (ey + kBrick - 1) / kBrick;
    const int snbz = (ez + kBrick - 1) / kBrick;
    const int b = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (b >= snbx * snby * snbz) return;
    const int lane = threadIdx.x & 31;
    const int sbx = b % snbx, sby = (b / snbx) % snby, sbz = b / (snbx * snby);
    const int x0 = sbx * kBrick, x1 = min(x0 + kBrick, ex) - 1;
    const int y0 = sby * kBrick, y1 = min(y0 + kBrick, ey) - 1;
    const int z0 = sbz * kBrick, z1 = min(z0 + kBrick, ez) - 1;
    const int x = x0 + (lane & 7), row = lane >> 3;
    uint32_t m0 = 0, m1 = 0, m2 = 0;
    if (x <= x1 && y0 + row <= y1) {
        const size_t plane = (size_t)ey * ex, step = 4 * (size_t)ex;
        const int nrows = (y1 - y0 - row) / 4 + 1;   // 1 or 2
        const unsigned char *q0 = lab + (size_t)z0 * plane + (size_t)(y0 + row) * ex + x;
        for (int z = z0; z <= z1; ++z, q0 += plane) {
            const unsigned char *q = q0;
            for (int r = 0; r < nrows; ++r, q += step) {
                int l = __ldg(q);
                if (l > 64) l = 64;
                if (l < 32) m0 |= 1u << l;
                else if (l < 64) m1 |= 1u << (l - 32);
                else m2 |= 1u;
            }
        }
    }
    m0 = __reduce_or_sync(0xffffffffu, m0);
    m1 = __reduce_or_sync(0xffffffffu, m1);
    m2 = __reduce_or_sync(0xffffffffu, m2);
    const size_t gb = ((size_t)(bz0 + sbz) * nby + (by0 + sby)) * nbx + (bx0 + sbx);
    if (lane < 3) {
        const uint32_t w = lane == 0 ? m0 : (lane == 1 ? m1 : m2);
        out[3 * gb + lane] = w;
        if (w) atomicOr(&present[lane], w);
    }
}

// Packed int16 min/max of 8 voxels of a row (uint4 of paired int16, SIMD
// vmins2/vmaxs2) plus the min/max of the row's two x-halo voxels, for the
// staged min/max kernel below; the label-set row kernel shares the brick-row
// decomposition: a block owns one brick row (blockIdx.x) for a run of kZRun
// z-bricks (blockIdx.y), thread t owns x-brick t.
constexpr int kZRun = 4;

struct Mm8 {
    uint4 lo, hi;      // packed int16 min / max over x = x0..x0+7
    int hlo, hhi;      // min / max of the x-halo voxels
};

__device__ __forceinline__ void mm8_init(Mm8 &m) {
    m.lo = make_uint4(0x7fff7fffu, 0x7fff7fffu, 0x7fff7fffu, 0x7fff7fffu);
    m.hi = make_uint4(0x80008000u, 0x80008000u, 0x80008000u, 0x80008000u);
    m.hlo = 32767;
    m.hhi = -32768;
}

__device__ __forceinline__ void mm8_merge(Mm8 &a, const Mm8 &b) {
    a.lo.x = __vmins2(a.lo.x, b.lo.x);
    a.lo.y = __vmins2(a.lo.y, b.lo.y);
    a.lo.z = __vmins2(a.lo.z, b.lo.z);
    a.lo.w = __vmins2(a.lo.w, b.lo.w);
    a.hi.x = __vmaxs2(a.hi.x, b.hi.x);
    a.hi.y = __vmaxs2(a.hi.y, b.hi.y);
    a.hi.z = __vmaxs2(a.hi.z, b.hi.z);
    a.hi.w = __vmaxs2(a.hi.w, b.hi.w);
    a.hlo = min(a.hlo, b.hlo);
    a.hhi = max(a.hhi, b.hhi);
}

__device__ __forceinline__ short2 mm8_result(const Mm8 &m) {
    uint32_t lo = __vmins2(__vmins2(m.lo.x, m.lo.y), __vmins2(m.lo.z, m.lo.w));
    uint32_t hi = __vmaxs2(__vmaxs2(m.hi.x, m.hi.y), __vmaxs2(m.hi.z, m.hi.w));
    const int l = min(min((int)(short)(lo & 0xffffu), (int)(short)(lo >> 16)), m.hlo);
    const int h = max(max((int)(short)(hi & 0xffffu), (int)(short)(hi >> 16)), m.hhi);
    return make_short2((short)l, (short)h);
}

// Label sets by rows: thread t owns x-brick t of one brick row for kZRun
// z-bricks, reads each 8-voxel row of its brick as one 8-byte word and sets
// one bit per distinct label (a row of one label, the common case, sets one
// bit).  The labels present anywhere in the volume are OR-ed into
// `present` (3 words) once per warp.
__device__ __forceinline__ void label_bits_word(uint32_t w, uint32_t &m0, uint32_t &m1, uint32_t &m2) {
    if (w == (w & 0xffu) * 0x01010101u) {
        int l = min((int)(w & 0xffu), 64);    // labels above MAXOBJECTCOUNT never occur via the API
        if (l < 32) m0 |= 1u << l;
        else if (l < 64) m1 |= 1u << (l - 32);
        else m2 |= 1u;
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int l = min((int)((w >> (8 * k)) & 0xffu), 64);
        if (l < 32) m0 |= 1u << l;
        else if (l < 64) m1 |= 1u << (l - 32);
        else m2 |= 1u;
    }
}

__global__ void __launch_bounds__(256) k_brick_labels_rows(const unsigned char *__restrict__ lab, int dx, int dy,
                                                            int dz, int nbx, int nby, int nbz, uint32_t *out,
                                                            uint32_t *present) {
    const int bx = threadIdx.x;
    uint32_t p0 = 0, p1 = 0, p2 = 0;
    if (bx < nbx) {
        const int by = blockIdx.x;
        const int bz0 = blockIdx.y * kZRun, bz1 = min(bz0 + kZRun, nbz);
        const int x0 = bx * kBrick;
        const int y0 = by * kBrick, ny = min(kBrick, dy - y0);
        const size_t plane = (size_t)dx * dy;
        for (int bz = bz0; bz < bz1; ++bz) {
            const int z0 = bz * kBrick, nz = min(kBrick, dz - z0);
            uint32_t m0 = 0, m1 = 0, m2 = 0;
            for (int z = z0; z < z0 + nz; ++z) {
                const unsigned char *base = lab + (size_t)z * plane + (size_t)y0 * dx + x0;
                uint2 w[kBrick];
#pragma unroll
                for (int r = 0; r < kBrick; ++r)
                    w[r] = r < ny ? __ldg(reinterpret_cast<const uint2 *>(base + (size_t)r * dx)) : w[0];
#pragma unroll
                for (int r = 0; r < kBrick; ++r) {
                    if (r < ny) {
                        label_bits_word(w[r].x, m0, m1, m2);
                        label_bits_word(w[r].y, m0, m1, m2);
                    }
                }
            }
            uint32_t *o = out + 3 * (((size_t)bz * nby + by) * nbx + bx);
            o[0] = m0;
            o[1] = m1;
            o[2] = m2;
            p0 |= m0;
            p1 |= m1;
            p2 |= m2;
        }
    }
    p0 = __reduce_or_sync(0xffffffffu, p0);
    p1 = __reduce_or_sync(0xffffffffu, p1);
    p2 = __reduce_or_sync(0xffffffffu, p2);
    if ((threadIdx.x & 31) == 0 && (p0 | p1 | p2)) {
        atomicOr(&present[0], p0);
        atomicOr(&present[1], p1);
        atomicOr(&present[2], p2);
    }
}

// ---------------------------------------------------------------------------
// Brick maps from slices staged in shared memory.  Each block (one brick row
// by, kZRun z-bricks) keeps kStages slices of its rows in flight: thread 0
// issues one bulk copy per row (cp.async.bulk, global -> shared, completion
// counted on the stage's mbarrier), every thread reads its brick's 16-byte
// row segment and both halo voxels from shared memory, and the stage is
// refilled with the slice kStages ahead once all threads have read it.  The
// loads of a block so run ahead of its arithmetic by kStages slices whatever
// the register count (kernels that load rows into registers wait on those
// loads: ncu showed long-scoreboard stalls).  Waits are bounded: a stage that
// does not complete within kStageWaitNs sets *err, and the block waits
// (bounded again) for its own copies before it returns.
constexpr int kStages = 4;
constexpr unsigned long long kStageWaitNs = 200ull * 1000 * 1000;   // 200 ms

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// 16-byte aligned source, destination and size
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// true once phase `parity` of the barrier has completed; false after
// kStageWaitNs (or 2^26 polls) without it
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < (1 << 26); ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 63) == 63 && global_ns() - t0 > kStageWaitNs) return false;
    }
    return false;
}

// Shared-memory bytes of the staged kernels: the barriers, then kStages
// slices of `rows` rows of `row_bytes`.
inline size_t staged_smem_bytes(int rows, size_t row_bytes) { return 128 + (size_t)kStages * rows * row_bytes; }

// The staged kernels apply when rows are whole bricks of 16-byte multiples
// and kStages slices fit in shared memory (dim_x up to about 2800).
bool brick_minmax_staged_fit(int dim_x, int nbx) {
    return dim_x % kBrick == 0 && nbx <= 256 && staged_smem_bytes(10, (size_t)dim_x * 2) <= 220 * 1024;
}
bool brick_labels_staged_fit(int dim_x, int nbx) {
    return dim_x % 16 == 0 && nbx <= 256 && staged_smem_bytes(8, (size_t)dim_x) <= 220 * 1024;
}

__global__ void __launch_bounds__(256) k_brick_minmax_staged(const short *__restrict__ vox, int dx, int dy, int dz,
                                                             int nbx, int nby, int nbz, short2 *out,
                                                             unsigned *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const short *stage0 = reinterpret_cast<const short *>(smem + 128);
    const size_t stage_elems = (size_t)10 * dx;
    const unsigned row_bytes = (unsigned)dx * 2;
    const int by = blockIdx.x;
    const int bz0 = blockIdx.y * kZRun, bz1 = min(bz0 + kZRun, nbz);
    const int za = max(bz0 * kBrick - 1, 0), zb = min(bz1 * kBrick, dz - 1);
    const int nsl = zb - za + 1;
    const size_t plane = (size_t)dx * dy;
    auto issue = [&](int st, int z) {        // thread 0: slice z into stage st
        uint64_t *bar = &bars[st];
        mbar_expect_tx(bar, 10u * row_bytes);
        unsigned char *dst = smem + 128 + (size_t)st * stage_elems * 2;
        for (int r = 0; r < 10; ++r) {
            const int y = min(max(by * kBrick - 1 + r, 0), dy - 1);
            bulk_to_smem(dst + (size_t)r * row_bytes, vox + (size_t)z * plane + (size_t)y * dx, row_bytes, bar);
        }
    };
    if (threadIdx.x == 0) {
        for (int st = 0; st < kStages; ++st) mbar_init(&bars[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < kStages && i < nsl; ++i) issue(i, za + i);
    const int lane = threadIdx.x & 31;
    const int bx = min((int)threadIdx.x, nbx - 1);
    const bool owner = (int)threadIdx.x < nbx;
    const int x0 = bx * kBrick;
    const bool left = bx > 0, right = bx + 1 < nbx;
    Mm8 acc, prev;
    mm8_init(acc);
    mm8_init(prev);
    int cur = bz0;
    bool failed = false;
    int i = 0;
    for (; i < nsl; ++i) {
        const int st = i % kStages;
        const bool ok = mbar_wait(&bars[st], (unsigned)(i / kStages) & 1u);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        const short *sl = stage0 + (size_t)st * stage_elems;
        Mm8 S;
        mm8_init(S);
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            const short *row = sl + (size_t)r * dx;
            const uint4 v = *reinterpret_cast<const uint4 *>(row + x0);
            S.lo.x = __vmins2(S.lo.x, v.x);
            S.lo.y = __vmins2(S.lo.y, v.y);
            S.lo.z = __vmins2(S.lo.z, v.z);
            S.lo.w = __vmins2(S.lo.w, v.w);
            S.hi.x = __vmaxs2(S.hi.x, v.x);
            S.hi.y = __vmaxs2(S.hi.y, v.y);
            S.hi.z = __vmaxs2(S.hi.z, v.z);
            S.hi.w = __vmaxs2(S.hi.w, v.w);
            // x halo from the neighbouring lanes (lanes 0 and 31 read it from the row)
            int l = (short)(__shfl_up_sync(0xffffffffu, v.w, 1) >> 16);
            int h = (short)(__shfl_down_sync(0xffffffffu, v.x, 1) & 0xffffu);
            if (lane == 0 && left) l = row[x0 - 1];
            if (lane == 31 && right) h = row[x0 + 8];
            if (!left) l = (short)(v.x & 0xffffu);
            if (!right) h = (short)(v.w >> 16);
            S.hlo = min(S.hlo, min(l, h));
            S.hhi = max(S.hhi, max(l, h));
        }
        __syncthreads();                      // every thread has read stage st
        if (threadIdx.x == 0 && i + kStages < nsl) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(st, za + i + kStages);
        }
        const int z = za + i;
        mm8_merge(acc, S);
        if ((z >> kBrickShift) > cur) {       // z = 8 (cur + 1): the slice above brick cur
            if (owner) out[((size_t)cur * nby + by) * nbx + bx] = mm8_result(acc);
            ++cur;
            acc = prev;                       // the slice below brick cur, then its first slice
            mm8_merge(acc, S);
        }
        prev = S;
    }
    if (failed) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1u);
            // copies in flight: stages i .. min(i + kStages, nsl) - 1; wait for them (bounded)
            for (int k = i; k < nsl && k < i + kStages; ++k) mbar_wait(&bars[k % kStages], (unsigned)(k / kStages) & 1u);
        }
        __syncthreads();
        return;
    }
    // the loop reads every issued slice (it stops at the slice above brick
    // bz1 - 1, the last one staged), so no copy is in flight here
    if (cur < bz1 && owner) out[((size_t)cur * nby + by) * nbx + bx] = mm8_result(acc);
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_brick_labels_staged(const unsigned char *__restrict__ lab, int dx, int dy,
                                                             int dz, int nbx, int nby, int nbz, uint32_t *out,
                                                             uint32_t *present, unsigned *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const size_t stage_bytes = (size_t)8 * dx;
    const int by = blockIdx.x;
    const int bz0 = blockIdx.y * kZRun, bz1 = min(bz0 + kZRun, nbz);
    const int z0 = bz0 * kBrick, z1 = min(bz1 * kBrick, dz);   // slices [z0, z1)
    const int nsl = z1 - z0;
    const int y0 = by * kBrick, ny = min(kBrick, dy - y0);
    const size_t plane = (size_t)dx * dy;
    auto issue = [&](int st, int z) {
        uint64_t *bar = &bars[st];
        mbar_expect_tx(bar, (unsigned)(ny * dx));
        unsigned char *dst = smem + 128 + (size_t)st * stage_bytes;
        for (int r = 0; r < ny; ++r)
            bulk_to_smem(dst + (size_t)r * dx, lab + (size_t)z * plane + (size_t)(y0 + r) * dx, (unsigned)dx, bar);
    };
    if (threadIdx.x == 0) {
        for (int st = 0; st < kStages; ++st) mbar_init(&bars[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < kStages && i < nsl; ++i) issue(i, z0 + i);
    const int bx = threadIdx.x;
    const bool owner = bx < nbx;
    const int x0 = (owner ? bx : 0) * kBrick;
    uint32_t m0 = 0, m1 = 0, m2 = 0, p0 = 0, p1 = 0, p2 = 0;
    bool failed = false;
    int i = 0;
    for (; i < nsl; ++i) {
        const int st = i % kStages;
        const bool ok = mbar_wait(&bars[st], (unsigned)(i / kStages) & 1u);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (owner) {
            const unsigned char *sl = smem + 128 + (size_t)st * stage_bytes;
            for (int r = 0; r < ny; ++r) {
                const uint2 w = *reinterpret_cast<const uint2 *>(sl + (size_t)r * dx + x0);
                label_bits_word(w.x, m0, m1, m2);
                label_bits_word(w.y, m0, m1, m2);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && i + kStages < nsl) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(st, z0 + i + kStages);
        }
        const int z = z0 + i;
        if (((z + 1) & (kBrick - 1)) == 0 || z + 1 == z1) {   // last slice of brick z >> 3
            if (owner) {
                uint32_t *o = out + 3 * (((size_t)(z >> kBrickShift) * nby + by) * nbx + bx);
                o[0] = m0;
                o[1] = m1;
                o[2] = m2;
            }
            p0 |= m0;
            p1 |= m1;
            p2 |= m2;
            m0 = m1 = m2 = 0;
        }
    }
    if (failed) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1u);
            for (int k = i; k < nsl && k < i + kStages; ++k) mbar_wait(&bars[k % kStages], (unsigned)(k / kStages) & 1u);
        }
        __syncthreads();
        return;
    }
    if (!owner) p0 = p1 = p2 = 0;
    p0 = __reduce_or_sync(0xffffffffu, p0);
    p1 = __reduce_or_sync(0xffffffffu, p1);
    p2 = __reduce_or_sync(0xffffffffu, p2);
    if ((threadIdx.x & 31) == 0 && (p0 | p1 | p2)) {
        atomicOr(&present[0], p0);
        atomicOr(&present[1], p1);
        atomicOr(&present[2], p2);
    }
}

__global__ void k_fill_labels_zero(uint32_t *out, int nbricks) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbricks) {
        out[3 * (size_t)b + 0] = 1u;   // label 0 only
        out[3 * (size_t)b + 1] = 0u;
        out[3 * (size_t)b + 2] = 0u;
    }
}

struct VisLabel {
    const float *lut_alpha;   // nullptr = no table
    int n;
    float alpha, ww, wl;
};

struct VisParams {
    VisLabel lab[MK_MAX_LABELS];
};

// One thread per brick.  VR: the brick is visible when, for some label it
// owns, the LUT alpha over the window of the brick's value range (widened by
// one LUT entry each side for the linear filter) exceeds kEmptyAlpha.  MIP:
// the largest windowed value (core/kernel.cu:339-345) over labels with
// alpha > 0.
__global__ void __launch_bounds__(256) k_brick_visibility(const short2 *__restrict__ minmax,
                                                          const uint32_t *__restrict__ labels,
                                                          int nbricks, VisParams P,
                                                          uint32_t *vis_bits, float *mip_tmax) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    bool vis = false;
    float tmax = -INFINITY;
    if (b < nbricks) {
        const short2 mm = minmax[b];
        // Normalized-float read of int16 is v/32767; the kernels scale it by
        // 32768 (core/kernel.cu:223).  Widen for the filter's rounding.
        const float k = 32768.0f / 32767.0f;
        const float hu_lo = (float)mm.x * k - (0.01f + 1e-5f * fabsf((float)mm.x));
        const float hu_hi = (float)mm.y * k + (0.01f + 1e-5f * fabsf((float)mm.y));
        for (int w = 0; w < 3; ++w) {
            uint32_t m = labels[3 * (size_t)b + w];
            while (m) {
                const int bit = __ffs(m) - 1;
                m &= m - 1;
                const int l = w * 32 + bit;
                if (l >= MK_MAX_LABELS) break;
                const VisLabel L = P.lab[l];
                const float t_lo = (hu_lo - L.wl) / L.ww + 0.5f;
                const float t_hi = (hu_hi - L.wl) / L.ww + 0.5f;
                if (L.alpha > 0.0f) tmax = fmaxf(tmax, t_hi);
                if (L.lut_alpha != nullptr && L.n > 0 && !vis) {
                    const float tl = fminf(t_lo, 1.0f), th = fminf(t_hi, 1.0f);
                    int i0 = (int)floorf(tl * L.n - 0.5f) - 1;
                    int i1 = (int)floorf(th * L.n - 0.5f) + 2;
                    if (!(tl == tl) || !(th == th)) {
                        i0 = 0;
                        i1 = L.n - 1;
                    }
                    i0 = max(0, min(i0, L.n - 1));
                    i1 = max(0, min(i1, L.n - 1));
                    for (int i = i0; i <= i1; ++i) {
                        if (L.lut_alpha[i] > kEmptyAlpha) {
                            vis = true;
                            break;
                        }
                    }
                }
            }
        }
        if (!(tmax == tmax)) tmax = INFINITY;
        mip_tmax[b] = tmax;
    }
    const uint32_t word = __ballot_sync(0xffffffffu, vis);
    if ((threadIdx.x & 31) == 0 && b < nbricks + 31) vis_bits[b >> 5] = word;
}

// The row kernels apply when every row splits into whole bricks and a block
// of one thread per x-brick stays within 256 threads.
bool brick_rows_fit(int dim_x, int nbx) { return dim_x % kBrick == 0 && nbx <= 256; }

int upload_linear(const void *host, size_t bytes, void **dptr, cudaStream_t s) {
    MK_CUDA_TRY(cudaMalloc(dptr, bytes));
    cudaError_t e = stage_to_device(*dptr, host, bytes, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(*dptr);
        *dptr = nullptr;
        set_last_error(std::string("upload: ") + cudaGetErrorString(e));
        return MK_ERR_CUDA;
    }
    return MK_OK;
}

int copy_to_array3d(const void *dsrc, size_t elem, int dx, int dy, int dz, cudaArray_t arr,
                     cudaStream_t s) {
    cudaMemcpy3DParms p;
    memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr(const_cast<void *>(dsrc), dx * elem, dx, dy);
    p.dstArray = arr;
    p.extent = make_cudaExtent(dx, dy, dz);
    p.kind = cudaMemcpyDeviceToDevice;
    MK_CUDA_TRY(cudaMemcpy3DAsync(&p, s));
    return MK_OK;
}

void free_tf(VolumeState &v, int l) {
    if (v.tf_tex[l]) cudaDestroyTextureObject(v.tf_tex[l]);
    if (v.tf_array[l]) cudaFreeArray(v.tf_array[l]);
    if (v.d_tf_alpha[l]) cudaFree(v.d_tf_alpha[l]);
    if (v.tf_len[l] > 0) v.device_bytes -= (size_t)v.tf_len[l] * 20;
    v.tf_tex[l] = 0;
    v.tf_array[l] = nullptr;
    v.d_tf_alpha[l] = nullptr;
    v.tf_len[l] = 0;
}

void free_mask(VolumeState &v) {
    if (v.tex_mask) cudaDestroyTextureObject(v.tex_mask);
    if (v.mask_array) {
        cudaFreeArray(v.mask_array);
        v.device_bytes -= (size_t)v.dims[0] * v.dims[1] * v.dims[2];
    }
    v.tex_mask = 0;
    v.mask_array = nullptr;
}

}  // namespace

float float_bound_above(double c) {
    float f = (float)c;
    if ((double)f <= c) f = nextafterf(f, INFINITY);
    return f;
}

BrickView brick_view(const VolumeState *v) {
    BrickView b;
    b.visible_bits = v->d_visible;
    b.mip_tmax = v->d_mip_tmax;
    b.minmax = v->d_minmax;
    b.nbx = v->nb[0];
    b.nby = v->nb[1];
    b.nbz = v->nb[2];
    return b;
}

LabelTable label_table(const VolumeState *v) {
    LabelTable t;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        t.tf[l] = v->tf_tex[l];
        t.alpha[l] = v->params[l][0];
        t.ww[l] = v->params[l][1];
        t.wl[l] = v->params[l][2];
    }
    return t;
}

int ensure_device_buffer(VolumeState *v, size_t bytes) {
    if (v->d_out_bytes >= bytes) return MK_OK;
    if (v->d_out) {
        cudaFree(v->d_out);
        v->device_bytes -= v->d_out_bytes;
        v->d_out = nullptr;
        v->d_out_bytes = 0;
    }
    MK_CUDA_TRY(cudaMalloc(&v->d_out, bytes));
    v->d_out_bytes = bytes;
    v->device_bytes += bytes;
    return MK_OK;
}

int ensure_pinned_buffer(VolumeState *v, size_t bytes) {
    if (v->h_pinned_bytes >= bytes) return MK_OK;
    if (v->h_pinned) {
        cudaFreeHost(v->h_pinned);
        v->h_pinned = nullptr;
        v->h_pinned_bytes = 0;
    }
    MK_CUDA_TRY(cudaMallocHost(&v->h_pinned, bytes));
    v->h_pinned_bytes = bytes;
    return MK_OK;
}

// Copy a finished device output to the caller.  Pinned (or registered)
// destinations receive the copy directly; pageable ones go through the
// volume's pinned staging buffer.
bool is_pinned_host(const void *p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess) return attr.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return false;
}

int finish_output(VolumeState *v, void *out, size_t bytes, int out_on_device, cudaStream_t s) {
    if (out_on_device) return MK_OK;
    const bool pinned = is_pinned_host(out);
    if (pinned) {
        MK_CUDA_TRY(cudaMemcpyAsync(out, v->d_out, bytes, cudaMemcpyDeviceToHost, s));
        MK_CUDA_TRY(cudaStreamSynchronize(s));
        return MK_OK;
    }
    int st = ensure_pinned_buffer(v, bytes);
    if (st != MK_OK) return st;
    MK_CUDA_TRY(cudaMemcpyAsync(v->h_pinned, v->d_out, bytes, cudaMemcpyDeviceToHost, s));
    MK_CUDA_TRY(cudaStreamSynchronize(s));
    memcpy(out, v->h_pinned, bytes);
    return MK_OK;
}

int launch_brick_visibility(const VolumeState *v, const float *const *lut_alpha, const int *lut_len,
                            const float (*params)[3], uint32_t *vis_bits, float *mip_tmax, cudaStream_t s) {
    const int nbricks = v->nb[0] * v->nb[1] * v->nb[2];
    VisParams P;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        P.lab[l].lut_alpha = lut_alpha[l];
        P.lab[l].n = lut_len[l];
        P.lab[l].alpha = params[l][0];
        P.lab[l].ww = params[l][1];
        P.lab[l].wl = params[l][2];
    }
    const int threads = 256;
    const int blocks = (nbricks + threads - 1) / threads;
    k_brick_visibility<<<blocks, threads, 0, s>>>(v->d_minmax, v->d_labels, nbricks, P, vis_bits, mip_tmax);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}

int rebuild_brick_maps(VolumeState *v, cudaStream_t s) {
    if (!v->maps_dirty) return MK_OK;
    const int rc = launch_brick_visibility(v, v->d_tf_alpha, v->tf_len, v->params, v->d_visible, v->d_mip_tmax, s);
    if (rc != MK_OK) return rc;
    v->maps_dirty = false;
    return MK_OK;
}

}  // namespace mk

using namespace mk;

extern "C" int mk_volume_create(mk_volume *out, const int16_t *voxels, int dim_x, int dim_y,
                                int dim_z, int device) {
    if (!out || !voxels || dim_x <= 0 || dim_y <= 0 || dim_z <= 0) {
        set_last_error("mk_volume_create: null pointer or non-positive dimension");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("mk_volume_create: no CUDA device");
        return MK_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) {
        set_last_error("mk_volume_create: device index out of range");
        return MK_ERR_INVALID_ARGUMENT;
    }
    DeviceGuard guard(device);
    mk_volume v = new mk_volume_s();
    VolumeState &st = v->st;
    st.device = device;
    st.dims[0] = dim_x;
    st.dims[1] = dim_y;
    st.dims[2] = dim_z;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        st.params[l][0] = 0.0f;   // AlphaAndWWWL() defaults (core/Defines.h:128-132), ww kept positive
        st.params[l][1] = 1.0f;
        st.params[l][2] = 0.0f;
    }
    int rc = MK_OK;
    void *d_lin = nullptr;
    const size_t nvox = (size_t)dim_x * dim_y * dim_z;
    do {
        if (cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_last_error("mk_volume_create: stream creation failed");
            rc = MK_ERR_CUDA;
            break;
        }
        rc = upload_linear(voxels, nvox * sizeof(short), &d_lin, st.stream);
        if (rc != MK_OK) break;

        cudaChannelFormatDesc cd = cudaCreateChannelDesc<short>();
        cudaError_t e = cudaMalloc3DArray(&st.vol_array, &cd, make_cudaExtent(dim_x, dim_y, dim_z));
        if (e != cudaSuccess) {
            set_last_error(std::string("cudaMalloc3DArray(volume): ") + cudaGetErrorString(e));
            rc = (e == cudaErrorMemoryAllocation) ? MK_ERR_OUT_OF_MEMORY : MK_ERR_CUDA;
            break;
        }
        st.device_bytes += nvox * sizeof(short);
        rc = copy_to_array3d(d_lin, sizeof(short), dim_x, dim_y, dim_z, st.vol_array, st.stream);
        if (rc != MK_OK) break;

        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = st.vol_array;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.normalizedCoords = 1;
        td.filterMode = cudaFilterModeLinear;
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.readMode = cudaReadModeNormalizedFloat;
        if (cudaCreateTextureObject(&st.tex_linear, &rd, &td, nullptr) != cudaSuccess) {
            set_last_error("mk_volume_create: linear texture creation failed");
            rc = MK_ERR_CUDA;
            break;
        }
        td.filterMode = cudaFilterModePoint;
        if (cudaCreateTextureObject(&st.tex_point, &rd, &td, nullptr) != cudaSuccess) {
            set_last_error("mk_volume_create: point texture creation failed");
            rc = MK_ERR_CUDA;
            break;
        }

        // brick maps
        st.nb[0] = (dim_x + kBrick - 1) / kBrick;
        st.nb[1] = (dim_y + kBrick - 1) / kBrick;
        st.nb[2] = (dim_z + kBrick - 1) / kBrick;
        const size_t nbricks = (size_t)st.nb[0] * st.nb[1] * st.nb[2];
        const size_t nwords = (nbricks + 31) / 32 + 1;
        if (cudaMalloc(&st.d_minmax, nbricks * sizeof(short2)) != cudaSuccess ||
            cudaMalloc(&st.d_labels, nbricks * 3 * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&st.d_visible, nwords * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&st.d_mip_tmax, nbricks * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&st.d_counter, sizeof(unsigned long long)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("mk_volume_create: brick map allocation failed");
            rc = MK_ERR_OUT_OF_MEMORY;
            break;
        }
        st.device_bytes += nbricks * (sizeof(short2) + 3 * sizeof(uint32_t) + sizeof(float)) +
                           nwords * sizeof(uint32_t) + sizeof(unsigned long long);
        cudaMemsetAsync(st.d_visible, 0, nwords * sizeof(uint32_t), st.stream);
        const bool staged = brick_minmax_staged_fit(dim_x, st.nb[0]);
        if (staged) {
            // d_counter doubles as the staged kernel's wait-timeout flag until the first render
            const size_t smem = staged_smem_bytes(10, (size_t)dim_x * 2);
            const dim3 grid(st.nb[1], (st.nb[2] + kZRun - 1) / kZRun);
            cudaMemsetAsync(st.d_counter, 0, sizeof(unsigned long long), st.stream);
            cudaFuncSetAttribute(k_brick_minmax_staged, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_brick_minmax_staged<<<grid, (st.nb[0] + 31) & ~31, smem, st.stream>>>(
                (const short *)d_lin, dim_x, dim_y, dim_z, st.nb[0], st.nb[1], st.nb[2], st.d_minmax,
                reinterpret_cast<unsigned *>(st.d_counter));
        } else {
            k_brick_minmax<<<(unsigned)((nbricks + 7) / 8), 256, 0, st.stream>>>(
                (const short *)d_lin, dim_x, dim_y, dim_z, st.nb[0], st.nb[1], (int)nbricks, st.d_minmax);
        }
        k_fill_labels_zero<<<(unsigned)((nbricks + 255) / 256), 256, 0, st.stream>>>(
            st.d_labels, (int)nbricks);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            set_last_error(std::string("brick map kernels: ") + cudaGetErrorString(e));
            rc = MK_ERR_CUDA;
            break;
        }

        // ray schedule table: a_{k+1} = fl(a_k + 1/dim_z) (core/kernel.cu:169, 213)
        const float step = 1.0f / (float)dim_z;
        const float limit = float_bound_above(1.732);
        std::vector<float> accu;
        accu.reserve((size_t)(1.74 * dim_z) + 8);
        float a = 0.0f;
        accu.push_back(a);
        while (a < limit) {
            a = a + step;
            accu.push_back(a);
        }
        st.accu_len = (int)accu.size();
        if (cudaMalloc(&st.d_accu, accu.size() * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("mk_volume_create: schedule table allocation failed");
            rc = MK_ERR_OUT_OF_MEMORY;
            break;
        }
        st.device_bytes += accu.size() * sizeof(float);
        e = cudaMemcpyAsync(st.d_accu, accu.data(), accu.size() * sizeof(float),
                            cudaMemcpyHostToDevice, st.stream);
        unsigned long long timed_out = 0;
        if (e == cudaSuccess && staged)
            e = cudaMemcpyAsync(&timed_out, st.d_counter, sizeof(timed_out), cudaMemcpyDeviceToHost, st.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st.stream);
        if (e != cudaSuccess) {
            set_last_error(std::string("mk_volume_create: ") + cudaGetErrorString(e));
            rc = MK_ERR_CUDA;
            break;
        }
        if (timed_out) {
            set_last_error("mk_volume_create: brick min/max staging timed out");
            rc = MK_ERR_TIMEOUT;
            break;
        }
    } while (0);
    if (d_lin) cudaFree(d_lin);
    if (rc != MK_OK) {
        mk_volume_destroy(v);
        return rc;
    }
    st.maps_dirty = true;
    *out = v;
    return MK_OK;
}

extern "C" int mk_volume_destroy(mk_volume v) {
    if (!v) return MK_ERR_INVALID_ARGUMENT;
    VolumeState &st = v->st;
    DeviceGuard guard(st.device);
    if (st.stream) cudaStreamSynchronize(st.stream);
    for (int l = 0; l < MK_MAX_LABELS; ++l) free_tf(st, l);
    free_mask(st);
    if (st.tex_linear) cudaDestroyTextureObject(st.tex_linear);
    if (st.tex_point) cudaDestroyTextureObject(st.tex_point);
    if (st.vol_array) cudaFreeArray(st.vol_array);
    cudaFree(st.d_minmax);
    cudaFree(st.d_labels);
    cudaFree(st.d_visible);
    cudaFree(st.d_mip_tmax);
    cudaFree(st.d_accu);
    cudaFree(st.d_out);
    cudaFree(st.d_counter);
    for (int i = 0; i < st.n_orders; ++i) {
        cudaFree(st.orders[i].d_tiles);
        if (st.orders[i].ready) cudaEventDestroy(st.orders[i].ready);
        free_table_uses(st.orders[i].uses);
    }
    for (int i = 0; i < st.n_tails; ++i) {
        cudaFree(st.tails[i].d_tail);
        cudaFree(st.tails[i].d_rays);
        if (st.tails[i].h_patch) cudaFreeHost(st.tails[i].h_patch);
        if (st.tails[i].copy_stream) cudaStreamDestroy(st.tails[i].copy_stream);
        if (st.tails[i].tiles_done) cudaEventDestroy(st.tails[i].tiles_done);
    }
    for (int i = 0; i < st.n_fy_tables; ++i) {
        cudaFree(st.fy_tables[i].d_fy);
        if (st.fy_tables[i].ready) cudaEventDestroy(st.fy_tables[i].ready);
        free_table_uses(st.fy_tables[i].uses);
    }
    cudaFree(st.d_voi_lut);
    if (st.voi_ready) cudaEventDestroy(st.voi_ready);
    free_table_uses(st.voi_uses);
    if (st.h_pinned) cudaFreeHost(st.h_pinned);
    if (st.stream) cudaStreamDestroy(st.stream);
    cudaGetLastError();
    delete v;
    return MK_OK;
}

extern "C" int mk_volume_device_bytes(mk_volume v, size_t *bytes) {
    if (!v || !bytes) return MK_ERR_INVALID_ARGUMENT;
    *bytes = v->st.device_bytes;
    return MK_OK;
}

extern "C" int mk_volume_brick_maps(mk_volume v, int *nb, int16_t *minmax, uint32_t *labels,
                                    uint64_t *present) {
    if (!v) {
        set_last_error("mk_volume_brick_maps: null volume");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &st = v->st;
    if (nb) {
        nb[0] = st.nb[0];
        nb[1] = st.nb[1];
        nb[2] = st.nb[2];
    }
    DeviceGuard guard(st.device);
    const size_t nbricks = brick_count(&st);
    if (minmax)
        MK_CUDA_TRY(cudaMemcpyAsync(minmax, st.d_minmax, nbricks * sizeof(short2), cudaMemcpyDeviceToHost,
                                    st.stream));
    if (labels)
        MK_CUDA_TRY(cudaMemcpyAsync(labels, st.d_labels, nbricks * 3 * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st.stream));
    MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
    if (present) {
        present[0] = st.present_labels[0];
        present[1] = st.present_labels[1];
    }
    return MK_OK;
}

extern "C" int mk_volume_dims(mk_volume v, int *dx, int *dy, int *dz) {
    if (!v || !dx || !dy || !dz) return MK_ERR_INVALID_ARGUMENT;
    *dx = v->st.dims[0];
    *dy = v->st.dims[1];
    *dz = v->st.dims[2];
    return MK_OK;
}

extern "C" int mk_volume_set_mask(mk_volume v, const uint8_t *labels) {
    if (!v) return MK_ERR_INVALID_ARGUMENT;
    VolumeState &st = v->st;
    DeviceGuard guard(st.device);
    const int dx = st.dims[0], dy = st.dims[1], dz = st.dims[2];
    const size_t nvox = (size_t)dx * dy * dz;
    const size_t nbricks = (size_t)st.nb[0] * st.nb[1] * st.nb[2];
    MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
    free_mask(st);
    st.maps_dirty = true;
    if (!labels) {
        st.present_labels[0] = 1;
        st.present_labels[1] = 0;
        k_fill_labels_zero<<<(unsigned)((nbricks + 255) / 256), 256, 0, st.stream>>>(st.d_labels,
                                                                                  (int)nbricks);
        MK_CUDA_TRY(cudaGetLastError());
        MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
        return MK_OK;
    }
    void *d_lin = nullptr;
    int rc = upload_linear(labels, nvox, &d_lin, st.stream);
    if (rc != MK_OK) return rc;
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<unsigned char>();
    cudaError_t e = cudaMalloc3DArray(&st.mask_array, &cd, make_cudaExtent(dx, dy, dz));
    if (e != cudaSuccess) {
        cudaFree(d_lin);
        set_last_error(std::string("cudaMalloc3DArray(mask): ") + cudaGetErrorString(e));
        return (e == cudaErrorMemoryAllocation) ? MK_ERR_OUT_OF_MEMORY : MK_ERR_CUDA;
    }
    st.device_bytes += nvox;
    rc = copy_to_array3d(d_lin, 1, dx, dy, dz, st.mask_array, st.stream);
    if (rc == MK_OK) {
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = st.mask_array;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.normalizedCoords = 0;
        td.filterMode = cudaFilterModePoint;
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.readMode = cudaReadModeElementType;
        if (cudaCreateTextureObject(&st.tex_mask, &rd, &td, nullptr) != cudaSuccess) {
            set_last_error("mk_volume_set_mask: texture creation failed");
            rc = MK_ERR_CUDA;
        }
    }
    // labels present anywhere (used to size per-ray state): OR-ed on the
    // device by the row kernel, else scanned on the host
    const bool rows = brick_rows_fit(dx, st.nb[0]);
    const bool staged = brick_labels_staged_fit(dx, st.nb[0]);
    uint32_t h_present[4] = {0, 0, 0, 0};   // label bits 0..64, then the staged kernel's timeout flag
    uint32_t *d_present = nullptr;
    if (rc == MK_OK && rows && cudaMalloc(&d_present, sizeof(h_present)) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("mk_volume_set_mask: allocation failed");
        rc = MK_ERR_OUT_OF_MEMORY;
    }
    if (rc == MK_OK) {
        if (rows) {
            e = cudaMemsetAsync(d_present, 0, sizeof(h_present), st.stream);
            const dim3 grid(st.nb[1], (st.nb[2] + kZRun - 1) / kZRun);
            if (e == cudaSuccess && staged) {
                const size_t smem = staged_smem_bytes(8, (size_t)dx);
                e = cudaFuncSetAttribute(k_brick_labels_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
                if (e == cudaSuccess)
                    k_brick_labels_staged<<<grid, (st.nb[0] + 31) & ~31, smem, st.stream>>>(
                        (const unsigned char *)d_lin, dx, dy, dz, st.nb[0], st.nb[1], st.nb[2], st.d_labels,
                        d_present, d_present + 3);
            } else if (e == cudaSuccess) {
                k_brick_labels_rows<<<grid, (st.nb[0] + 31) & ~31, 0, st.stream>>>(
                    (const unsigned char *)d_lin, dx, dy, dz, st.nb[0], st.nb[1], st.nb[2], st.d_labels, d_present);
            }
        } else {
            k_brick_labels<<<(unsigned)((nbricks + 7) / 8), 256, 0, st.stream>>>(
                (const unsigned char *)d_lin, dx, dy, dz, st.nb[0], st.nb[1], (int)nbricks, st.d_labels);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess && rows)
            e = cudaMemcpyAsync(h_present, d_present, sizeof(h_present), cudaMemcpyDeviceToHost, st.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st.stream);
        if (e != cudaSuccess) {
            set_last_error(std::string("mk_volume_set_mask: ") + cudaGetErrorString(e));
            rc = MK_ERR_CUDA;
        } else if (h_present[3]) {
            set_last_error("mk_volume_set_mask: brick label staging timed out");
            rc = MK_ERR_TIMEOUT;
        }
    }
    cudaFree(d_present);
    cudaFree(d_lin);
    if (rc != MK_OK) {
        free_mask(st);
        return rc;
    }
    uint64_t pres[2] = {0, 0};
    if (rows) {
        pres[0] = (uint64_t)h_present[0] | ((uint64_t)h_present[1] << 32);
        pres[1] = h_present[2] & 1u;
    } else {
        for (size_t i = 0; i < nvox; ++i) {
            const int l = labels[i] > 64 ? 64 : labels[i];
            pres[l >> 6] |= 1ull << (l & 63);
        }
    }
    st.present_labels[0] = pres[0];
    st.present_labels[1] = pres[1];
    return MK_OK;
}

extern "C" int mk_volume_update_mask(mk_volume v, const uint8_t *labels, const int box[6]) {
    if (!v || !labels || !box) {
        set_last_error("mk_volume_update_mask: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &st = v->st;
    if (!st.mask_array) {
        set_last_error("mk_volume_update_mask: the volume has no mask (use mk_volume_set_mask)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const int dx = st.dims[0], dy = st.dims[1], dz = st.dims[2];
    const int lo[3] = {box[0], box[1], box[2]}, hi[3] = {box[3], box[4], box[5]};
    const int dim[3] = {dx, dy, dz};
    for (int k = 0; k < 3; ++k) {
        if (lo[k] < 0 || hi[k] > dim[k] || lo[k] >= hi[k]) {
            set_last_error("mk_volume_update_mask: box outside the volume or empty");
            return MK_ERR_INVALID_ARGUMENT;
        }
    }
    // widen to whole bricks (clamped to the volume): a brick's label set
    // depends on its own voxels only
    int b0[3], e[3];
    for (int k = 0; k < 3; ++k) {
        b0[k] = lo[k] & ~(kBrick - 1);
        e[k] = std::min((hi[k] + kBrick - 1) & ~(kBrick - 1), dim[k]) - b0[k];
    }
    DeviceGuard guard(st.device);
    // the array is written in place: renders of this volume on any stream
    // must have finished reading it
    MK_CUDA_TRY(cudaDeviceSynchronize());
    const size_t sub = (size_t)e[0] * e[1] * e[2];
    unsigned char *d_sub = nullptr;
    uint32_t *d_present = nullptr;
    if (cudaMalloc(&d_sub, sub) != cudaSuccess || cudaMalloc(&d_present, 3 * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_sub);
        set_last_error("mk_volume_update_mask: allocation failed");
        return MK_ERR_OUT_OF_MEMORY;
    }
    uint32_t h_present[3] = {0, 0, 0};
    cudaError_t err = cudaMemsetAsync(d_present, 0, 3 * sizeof(uint32_t), st.stream);
    // host box -> linear device box -> the mask array at the box's place
    cudaMemcpy3DParms hp;
    memset(&hp, 0, sizeof(hp));
    hp.srcPtr = make_cudaPitchedPtr(const_cast<uint8_t *>(labels), dx, dx, dy);
    hp.srcPos = make_cudaPos(b0[0], b0[1], b0[2]);
    hp.dstPtr = make_cudaPitchedPtr(d_sub, e[0], e[0], e[1]);
    hp.extent = make_cudaExtent(e[0], e[1], e[2]);
    hp.kind = cudaMemcpyHostToDevice;
    if (err == cudaSuccess) err = cudaMemcpy3DAsync(&hp, st.stream);
    cudaMemcpy3DParms ap;
    memset(&ap, 0, sizeof(ap));
    ap.srcPtr = make_cudaPitchedPtr(d_sub, e[0], e[0], e[1]);
    ap.dstArray = st.mask_array;
    ap.dstPos = make_cudaPos(b0[0], b0[1], b0[2]);
    ap.extent = make_cudaExtent(e[0], e[1], e[2]);
    ap.kind = cudaMemcpyDeviceToDevice;
    if (err == cudaSuccess) err = cudaMemcpy3DAsync(&ap, st.stream);
    if (err == cudaSuccess) {
        const int nsub = ((e[0] + kBrick - 1) / kBrick) * ((e[1] + kBrick - 1) / kBrick) *
                         ((e[2] + kBrick - 1) / kBrick);
        k_brick_labels_box<<<(unsigned)((nsub + 7) / 8), 256, 0, st.stream>>>(
            d_sub, e[0], e[1], e[2], b0[0] / kBrick, b0[1] / kBrick, b0[2] / kBrick, st.nb[0], st.nb[1],
            st.d_labels, d_present);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(h_present, d_present, sizeof(h_present), cudaMemcpyDeviceToHost, st.stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st.stream);
    cudaFree(d_sub);
    cudaFree(d_present);
    if (err != cudaSuccess) {
        set_last_error(std::string("mk_volume_update_mask: ") + cudaGetErrorString(err));
        return MK_ERR_CUDA;
    }
    // labels can only be added to the set here (see the header)
    st.present_labels[0] |= (uint64_t)h_present[0] | ((uint64_t)h_present[1] << 32);
    st.present_labels[1] |= h_present[2] & 1u;
    st.maps_dirty = true;
    return MK_OK;
}

extern "C" int mk_volume_set_transfer_function(mk_volume v, int label, const float *rgba,
                                               int n_entries) {
    if (!v || label < 0 || label >= MK_MAX_LABELS) {
        set_last_error("mk_volume_set_transfer_function: bad volume or label");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &st = v->st;
    DeviceGuard guard(st.device);
    MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
    st.maps_dirty = true;
    if (rgba && n_entries > 0 && n_entries == st.tf_len[label] && st.tf_array[label]) {
        // same length: overwrite the table in place (the texture object stays valid)
        std::vector<float> alpha(n_entries);
        for (int i = 0; i < n_entries; ++i) alpha[i] = rgba[4 * i + 3];
        // on the volume's stream (a plain cudaMemcpy from pageable memory may
        // return before the data lands, unordered with this non-blocking stream)
        MK_CUDA_TRY(cudaMemcpy2DToArrayAsync(st.tf_array[label], 0, 0, rgba, n_entries * sizeof(float4),
                                             n_entries * sizeof(float4), 1, cudaMemcpyHostToDevice, st.stream));
        MK_CUDA_TRY(cudaMemcpyAsync(st.d_tf_alpha[label], alpha.data(), n_entries * sizeof(float),
                                    cudaMemcpyHostToDevice, st.stream));
        MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
        return MK_OK;
    }
    free_tf(st, label);
    if (!rgba || n_entries <= 0) return MK_OK;   // label becomes transparent
    if (n_entries > 65536) {
        set_last_error("mk_volume_set_transfer_function: more than 65536 entries");
        return MK_ERR_INVALID_ARGUMENT;
    }
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
    MK_CUDA_TRY(cudaMallocArray(&st.tf_array[label], &cd, n_entries, 1));
    MK_CUDA_TRY(cudaMemcpy2DToArrayAsync(st.tf_array[label], 0, 0, rgba, n_entries * sizeof(float4),
                                         n_entries * sizeof(float4), 1, cudaMemcpyHostToDevice, st.stream));
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = st.tf_array[label];
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.normalizedCoords = 1;
    td.filterMode = cudaFilterModeLinear;
    td.addressMode[0] = cudaAddressModeClamp;
    td.readMode = cudaReadModeElementType;
    MK_CUDA_TRY(cudaCreateTextureObject(&st.tf_tex[label], &rd, &td, nullptr));
    std::vector<float> alpha(n_entries);
    for (int i = 0; i < n_entries; ++i) alpha[i] = rgba[4 * i + 3];
    MK_CUDA_TRY(cudaMalloc(&st.d_tf_alpha[label], n_entries * sizeof(float)));
    MK_CUDA_TRY(cudaMemcpyAsync(st.d_tf_alpha[label], alpha.data(), n_entries * sizeof(float),
                                cudaMemcpyHostToDevice, st.stream));
    MK_CUDA_TRY(cudaStreamSynchronize(st.stream));
    st.tf_len[label] = n_entries;
    st.device_bytes += (size_t)n_entries * 20;
    return MK_OK;
}

extern "C" int mk_volume_set_label_params(mk_volume v, const float *alpha_ww_wl, int n_labels) {
    if (!v || !alpha_ww_wl || n_labels <= 0 || n_labels > MK_MAX_LABELS) {
        set_last_error("mk_volume_set_label_params: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    for (int l = 0; l < n_labels; ++l) {
        if (!(alpha_ww_wl[3 * l + 1] > 0.0f)) {
            set_last_error("mk_volume_set_label_params: window width must be > 0");
            return MK_ERR_INVALID_ARGUMENT;
        }
    }
    VolumeState &st = v->st;
    for (int l = 0; l < n_labels; ++l) {
        st.params[l][0] = alpha_ww_wl[3 * l + 0];
        st.params[l][1] = alpha_ww_wl[3 * l + 1];
        st.params[l][2] = alpha_ww_wl[3 * l + 2];
    }
    st.maps_dirty = true;
    return MK_OK;
}

extern "C" int mk_volume_synchronize(mk_volume v, void *stream) {
    if (!v) return MK_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(v->st.device);
    cudaStream_t s = stream ? (cudaStream_t)stream : v->st.stream;
    MK_CUDA_TRY(cudaStreamSynchronize(s));
    return MK_OK;
}
