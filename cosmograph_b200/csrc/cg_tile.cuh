// cg_tile.cuh -- periodic halo tiles of one field in shared memory, shared by
// the FP64 and FP32-mixed substep kernels.
//
// A CTA owns a brick of BX x BY x BZ points (x, y, z), one point per thread,
// z fastest.  For each field whose derivatives the point needs, the CTA
// copies the brick plus an r = O/2 halo on every side (periodic wrap applied
// at the copy) into shared memory once; every stencil tap is then a
// shared-memory load at a compile-time offset from the thread's centre.
//
// Bricks and row pitches are chosen so that a warp's tap is free of bank
// conflicts:
//   FP64, 4 x 2 x 16: a warp reads two contiguous 16-double rows (two
//         wavefronts, the minimum for 256 bytes);
//   FP32, 4 x 4 x 8 with a row pitch of 24 floats: a warp reads four 8-float
//         row segments whose banks are s, s+24, s+16, s+8 (mod 32), one
//         wavefront.
//
// The copy is software-pipelined by the caller: the next field's elements are
// fetched into registers while the current tile is being read (Loader), or,
// with a second tile buffer, copied by cp.async straight into it
// (AsyncLoader).
#pragma once

namespace cg {
namespace tile {

template <int BX_, int BY_, int BZ_>
struct Brick {
  static constexpr int BX = BX_, BY = BY_, BZ = BZ_, THREADS = BX * BY * BZ, WARPS = THREADS / 32;
};
using Brick64 = Brick<4, 2, 16>;
using Brick32 = Brick<4, 4, 8>;

// PITCH: row pitch in elements (0: the copied row length).  ZOFF: tile
// column 0 holds z = z0 - ZOFF (default r); the copy fills columns
// CO = ZOFF - r ... CO + BZ + 2r - 1.  A tile filled by a TMA box starts at
// an aligned z, below the halo.
template <int O, class B, int PITCH = 0, int ZOFF = -1>
struct Geom {
  static constexpr int R = O / 2;
  static constexpr int ZO = ZOFF < 0 ? R : ZOFF;          // tile column 0: z = z0 - ZO
  static constexpr int CO = ZO - R;                        // first copied column
  static constexpr int TX = B::BX + 2 * R, TY = B::BY + 2 * R;
  static constexpr int TZU = B::BZ + 2 * R;                // z values copied per row
  static constexpr int TZ = PITCH ? PITCH : TZU;           // row pitch
  static_assert(CO >= 0 && CO + TZU <= TZ, "a row holds the brick and its halo");
  static constexpr int ROWS = TX * TY;
  static constexpr int SIZE = ROWS * TZ;
  static constexpr int SY = TZ, SX = TY * TZ;
  static constexpr int RPP = 32 / TZU;                    // rows per warp instruction
  static constexpr int NPW = (ROWS + B::WARPS * RPP - 1) / (B::WARPS * RPP);  // instructions per warp
  static_assert(TZU <= 32, "one warp copies at least one tile row");
};

// v mod n in [0, n) for any v (tile coordinates reach past one period on
// boxes smaller than the halo)
__device__ __forceinline__ int pmod(int v, int n) {
  const int r = v % n;
  return r < 0 ? r + n : r;
}

// Global offset of the first element of each tile row, row r = x*TY + y of
// the brick at (x0, y0): ((x0 - R + x) mod nx, (y0 - R + y) mod ny) * nz.
// Written by threads r; the caller synchronises the CTA before any Loader
// reads them.
template <class G, class B>
__device__ __forceinline__ void row_offsets(int x0, int y0, int nx, int ny, int nz, int tid, int* rowoff) {
  for (int r = tid; r < G::ROWS; r += B::THREADS) {
    const int x = pmod(x0 - G::R + r / G::TY, nx), y = pmod(y0 - G::R + r % G::TY, ny);
    rowoff[r] = (x * ny + y) * nz;
  }
}

// Copy of one field's tile.  Lane l of warp w works on column z = l mod TZU of
// row (w + WARPS*q)*RPP + l / TZU at step q.  fetch() issues the global loads
// into registers, store() writes them to the tile.
template <class G, class B, class T>
struct Loader {
  T buf[G::NPW];
  int row0, col, zoff;  // zoff < 0: lane without a column
  __device__ __forceinline__ void init(int tid, int z0, int nz) {
    const int warp = tid >> 5, lane = tid & 31;
    const int sub = lane / G::TZU;
    col = lane - sub * G::TZU;
    row0 = warp * G::RPP + sub;
    zoff = sub < G::RPP ? pmod(z0 - G::R + col, nz) : -1;
  }
  __device__ __forceinline__ void fetch(const T* __restrict__ f, const int* rowoff) {
#pragma unroll
    for (int q = 0; q < G::NPW; ++q) {
      const int r = row0 + B::WARPS * G::RPP * q;
      if (zoff >= 0 && r < G::ROWS) buf[q] = __ldg(f + rowoff[r] + zoff);
    }
  }
  __device__ __forceinline__ void store(T* tl) const {
#pragma unroll
    for (int q = 0; q < G::NPW; ++q) {
      const int r = row0 + B::WARPS * G::RPP * q;
      if (zoff >= 0 && r < G::ROWS) tl[r * G::TZ + G::CO + col] = buf[q];
    }
  }
};

// Asynchronous copy of one field's tile (cp.async, global to shared memory,
// no register staging), with the lane/row mapping of Loader.  issue() starts
// this thread's copies and commits them as one group; the caller waits for
// its groups (cp_async_wait) and synchronises the CTA before reading.
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <class G, class B>
struct AsyncLoader {
  int row0, col, zoff;  // zoff < 0: lane without a column
  __device__ __forceinline__ void init(int tid, int z0, int nz) {
    const int warp = tid >> 5, lane = tid & 31;
    const int sub = lane / G::TZU;
    col = lane - sub * G::TZU;
    row0 = warp * G::RPP + sub;
    zoff = sub < G::RPP ? pmod(z0 - G::R + col, nz) : -1;
  }
  __device__ __forceinline__ void issue(double* tl, const double* __restrict__ f, const int* rowoff) const {
#pragma unroll
    for (int q = 0; q < G::NPW; ++q) {
      const int r = row0 + B::WARPS * G::RPP * q;
      if (zoff >= 0 && r < G::ROWS) cp_async(tl + r * G::TZ + G::CO + col, f + rowoff[r] + zoff);
    }
    cp_async_commit();
  }
};

// Stencil taps of one thread's point in a tile: values at offsets n along
// axis a, or (n, m) along axes (a, b).
template <class G, class T>
struct Taps {
  const T* t;
  int cc;  // the centre's tile index
  __device__ __forceinline__ static int off(int a, int n) { return a == 0 ? n * G::SX : (a == 1 ? n * G::SY : n); }
  __device__ __forceinline__ T ax(int a, int n) const { return t[cc + off(a, n)]; }
  __device__ __forceinline__ T pl(int a, int n, int b, int m) const { return t[cc + off(a, n) + off(b, m)]; }
};

// tile index of the centre of thread (tx, ty, tz) = (threadIdx.z, .y, .x)
template <class G>
__device__ __forceinline__ int centre(int tx, int ty, int tz) {
  return ((tx + G::R) * G::TY + (ty + G::R)) * G::TZ + (tz + G::ZO);
}

}  // namespace tile
}  // namespace cg
