// Device helpers of the octree build shared by the single-tree build (nb_tree.cu) and the
// batched forest build (nb_batch.cu).  Included only by translation units compiled with
// -fmad=false: the floating-point expressions keep the reference's rounding.  Bare line
// citations (:N) refer to nbody/src/nbody_tree.c.
#pragma once
#include "nb_common.cuh"

__device__ __forceinline__ long long nb_grid(double x, double scale)
{
    // CPU: a NaN coordinate fails every `mid <= pos`, i.e. it always takes the lower child.
    if (isnan(x)) return 0;
    double f = floor(x * scale);
    long long k = (long long) f + (1ll << (NB_GRID_LEVELS - 1));
    if (k < 0) k = 0;
    if (k > (1ll << NB_GRID_LEVELS) - 1) k = (1ll << NB_GRID_LEVELS) - 1;
    return k;
}

__device__ __forceinline__ unsigned long long nb_spread21(unsigned long long v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// x is the most significant bit of each octant triplet: the child index of nbSubIndex
// is 4*[x] + 2*[y] + [z] (:36-52), so key order is the CPU's child order at every level.
__device__ __forceinline__ unsigned long long nb_morton63(long long kx, long long ky, long long kz)
{
    const int sh = NB_GRID_LEVELS - NB_KEY_LEVELS;
    return (nb_spread21((unsigned long long) kx >> sh) << 2) |
           (nb_spread21((unsigned long long) ky >> sh) << 1) |
            nb_spread21((unsigned long long) kz >> sh);
}

// Morton order of two full 62-level paths: the first differing level decides, and within
// it x outranks y outranks z (child index 4x+2y+z).
__device__ __forceinline__ bool nb_path_less(long long ax, long long ay, long long az,
                                             long long bx, long long by, long long bz)
{
    const unsigned long long dx = (unsigned long long) (ax ^ bx);
    const unsigned long long dy = (unsigned long long) (ay ^ by);
    const unsigned long long dz = (unsigned long long) (az ^ bz);
    const int hx = dx ? 63 - __clzll(dx) : -1;
    const int hy = dy ? 63 - __clzll(dy) : -1;
    const int hz = dz ? 63 - __clzll(dz) : -1;
    if (hx < 0 && hy < 0 && hz < 0) return false;
    if (hx >= hy && hx >= hz) return ax < bx;
    if (hy >= hz) return ay < by;
    return az < bz;
}

__device__ __forceinline__ int nb_part_depth(long long ax, long long ay, long long az,
                                             long long bx, long long by, long long bz)
{
    unsigned long long d = (unsigned long long) ((ax ^ bx) | (ay ^ by) | (az ^ bz));
    if (d == 0) return NB_GRID_LEVELS;            // same point on the grid
    return (NB_GRID_LEVELS - 1) - (63 - __clzll(d));
}

// Last sorted body sharing the depth-D path prefix of body a (bodies of one cell are
// contiguous in path order): galloping then binary search.
__device__ inline int nb_range_end(const long long* gx, const long long* gy, const long long* gz,
                            int a, int D, int m)
{
    if (D == 0) return m - 1;
    const int s = NB_GRID_LEVELS - D;
    const long long ax = gx[a] >> s, ay = gy[a] >> s, az = gz[a] >> s;
    int lo = a, step = 1;
    while (lo + step < m && (gx[lo + step] >> s) == ax && (gy[lo + step] >> s) == ay &&
           (gz[lo + step] >> s) == az) {
        lo += step;
        step <<= 1;
    }
    int hi = min(lo + step, m);          // first index known (or assumed) outside
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((gx[mid] >> s) == ax && (gy[mid] >> s) == ay && (gz[mid] >> s) == az) lo = mid;
        else hi = mid;
    }
    return lo;
}

// findRCrit (:308-343) from the cell's geometric centre, CoM and size.
__device__ __forceinline__ double nb_find_rcrit2(int criterion, double theta, double rsize,
                                                 double cx, double cy, double cz,
                                                 double mx, double my, double mz, double psize)
{
    if (theta == 0.0) {
        const double rc = 2.0 * rsize;
        return rc * rc;
    }
    switch (criterion) {
    case NBCUDA_TREECODE: {
        const double dx = mx - cx, dy = my - cy, dz = mz - cz;
        const double rc = psize / theta + sqrt(dx * dx + dy * dy + dz * dz);
        return rc * rc;
    }
    case NBCUDA_SW93: {
        double dmin, b, bmax2;
        dmin = mx - (cx - 0.5 * psize); b = fmax(dmin, psize - dmin); bmax2 = b * b;
        dmin = my - (cy - 0.5 * psize); b = fmax(dmin, psize - dmin); bmax2 += b * b;
        dmin = mz - (cz - 0.5 * psize); b = fmax(dmin, psize - dmin); bmax2 += b * b;
        return bmax2 / (theta * theta);
    }
    case NBCUDA_BH86: {
        const double rc = psize / theta;
        return rc * rc;
    }
    default:
        return 0.0;
    }
}

// L2 loads (bypass L1: cells computed by other blocks in this kernel must not be read
// from a stale L1 line)
__device__ __forceinline__ double4 nb_ld_pm(const double4* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

