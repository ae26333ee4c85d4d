// tw_synth.cpp -- a procedural tile source and a checksum tile sink, so that
// the tiled path can be run at the terabyte scale of its largest workload
// (16384 x 16384 x 4096 uint16) with no volume stored anywhere.
//
// A 256^3 base block is generated once per (seed, type) from a seeded
// integer hash: noise 0..10, Gaussian blobs (sigma 2-8 voxels, peaks
// 400-4095 for uint16, 40-255 for uint8; about one per 64^3 cell, each
// cell's blobs drawn from a hash of the cell) and short one-voxel-wide
// random-walk fibres (values 2500-4095 / 200-255).  Voxel (x, y, z) of the
// volume is the base block's voxel shifted cyclically by an offset hashed
// from the 512^3 tile that contains (x, y, z): every tile looks different,
// every voxel is a function of its coordinates and the seed alone (two boxes
// agree where they overlap), and a box is read with a few memory copies per
// row, fast enough to feed the GPU.
#include "tw_host.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr int kCell = 64;        // blob / fibre cells
constexpr int kMaxBlobs = 3;     // per cell
constexpr int kReach = 24;       // 3 sigma of the widest blob
constexpr int kFibreSteps = 48;  // fibre length (voxels)

inline uint64_t mix(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

inline uint64_t hash4(uint64_t seed, int64_t a, int64_t b, int64_t c, uint64_t k)
{
    return mix(seed * 0x9E3779B97F4A7C15ULL ^ mix((uint64_t)a * 0xA24BAED4963EE407ULL ^
                                                 mix((uint64_t)b * 0x9FB21C651E98DF25ULL ^
                                                     mix((uint64_t)c * 0xD6E8FEB86659FD93ULL ^ k))));
}

inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Blob {
    double c[3], sigma, peak;
};

// The blobs of cell (cx, cy, cz), in a fixed order.
int cell_blobs(uint64_t seed, int64_t cx, int64_t cy, int64_t cz, bool u16, Blob out[kMaxBlobs])
{
    const uint64_t h = hash4(seed, cx, cy, cz, 1);
    const int n = (int)(h % 4) == 3 ? 2 : (int)(h % 4) % 2;  // 0, 1, 0, 2 blobs: ~0.75 per cell
    for (int i = 0; i < n; ++i) {
        const uint64_t k = 16 + 8 * (uint64_t)i;
        out[i].c[0] = (double)(cx * kCell) + unit(hash4(seed, cx, cy, cz, k)) * kCell;
        out[i].c[1] = (double)(cy * kCell) + unit(hash4(seed, cx, cy, cz, k + 1)) * kCell;
        out[i].c[2] = (double)(cz * kCell) + unit(hash4(seed, cx, cy, cz, k + 2)) * kCell;
        out[i].sigma = 2.0 + 6.0 * unit(hash4(seed, cx, cy, cz, k + 3));
        out[i].peak = u16 ? 400.0 + 3695.0 * unit(hash4(seed, cx, cy, cz, k + 4))
                          : 40.0 + 215.0 * unit(hash4(seed, cx, cy, cz, k + 4));
    }
    return n;
}

inline int64_t fdiv(int64_t a, int64_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

struct Gen {
    uint64_t seed;
    int dtype;
};

// Fills planes [z0, z1) of the box (x0, y0, nx, ny) of the hash-generated
// field into dst (pitch nx, nx*ny).
void fill_slab(const Gen *v, int64_t x0, int64_t y0, int64_t z0, int64_t z1, int64_t nx, int64_t ny,
               void *dst_box, int64_t zbox0)
{
    const bool u16 = v->dtype == TW_U16;
    const double vmax = u16 ? 4095.0 : 255.0;
    const int64_t nz = z1 - z0;
    std::vector<float> acc((size_t)(nx * ny * nz));
    // noise 0..10 from a hash of the global index
    for (int64_t z = z0; z < z1; ++z)
        for (int64_t y = y0; y < y0 + ny; ++y) {
            float *row = acc.data() + ((z - z0) * ny + (y - y0)) * nx;
            for (int64_t x = x0; x < x0 + nx; ++x)
                row[x - x0] = (float)(hash4(v->seed, x, y, z, 7) % 11);
        }
    // blobs of every cell within reach, in cell order
    const int64_t c0[3] = {fdiv(x0 - kReach, kCell), fdiv(y0 - kReach, kCell), fdiv(z0 - kReach, kCell)};
    const int64_t c1[3] = {fdiv(x0 + nx - 1 + kReach, kCell), fdiv(y0 + ny - 1 + kReach, kCell),
                           fdiv(z1 - 1 + kReach, kCell)};
    std::vector<float> gx, gy, gz;
    for (int64_t cz = c0[2]; cz <= c1[2]; ++cz)
        for (int64_t cy = c0[1]; cy <= c1[1]; ++cy)
            for (int64_t cx = c0[0]; cx <= c1[0]; ++cx) {
                Blob b[kMaxBlobs];
                const int n = cell_blobs(v->seed, cx, cy, cz, u16, b);
                for (int i = 0; i < n; ++i) {
                    const int64_t r = (int64_t)std::ceil(3.0 * b[i].sigma);
                    const int64_t lo[3] = {std::max(x0, (int64_t)b[i].c[0] - r), std::max(y0, (int64_t)b[i].c[1] - r),
                                           std::max(z0, (int64_t)b[i].c[2] - r)};
                    const int64_t hi[3] = {std::min(x0 + nx, (int64_t)b[i].c[0] + r + 1),
                                           std::min(y0 + ny, (int64_t)b[i].c[1] + r + 1),
                                           std::min(z1, (int64_t)b[i].c[2] + r + 1)};
                    if (lo[0] >= hi[0] || lo[1] >= hi[1] || lo[2] >= hi[2]) continue;
                    const double inv = -0.5 / (b[i].sigma * b[i].sigma);
                    auto fac = [&](std::vector<float> &g, int a) {
                        g.resize((size_t)(hi[a] - lo[a]));
                        for (int64_t t = lo[a]; t < hi[a]; ++t) {
                            const double d = (double)t - b[i].c[a];
                            g[(size_t)(t - lo[a])] = (float)std::exp(d * d * inv);
                        }
                    };
                    fac(gx, 0);
                    fac(gy, 1);
                    fac(gz, 2);
                    const float pk = (float)b[i].peak;
                    for (int64_t z = lo[2]; z < hi[2]; ++z)
                        for (int64_t y = lo[1]; y < hi[1]; ++y) {
                            const float wzy = pk * gz[(size_t)(z - lo[2])] * gy[(size_t)(y - lo[1])];
                            float *row = acc.data() + ((z - z0) * ny + (y - y0)) * nx - x0;
                            for (int64_t x = lo[0]; x < hi[0]; ++x) row[x] += wzy * gx[(size_t)(x - lo[0])];
                        }
                }
            }
    // fibres: a walk of kFibreSteps voxels from a hashed start in one cell of
    // eight; each visited voxel takes the fibre's value
    const int64_t f0[3] = {fdiv(x0 - kFibreSteps, kCell), fdiv(y0 - kFibreSteps, kCell), fdiv(z0 - kFibreSteps, kCell)};
    const int64_t f1[3] = {fdiv(x0 + nx - 1 + kFibreSteps, kCell), fdiv(y0 + ny - 1 + kFibreSteps, kCell),
                           fdiv(z1 - 1 + kFibreSteps, kCell)};
    for (int64_t cz = f0[2]; cz <= f1[2]; ++cz)
        for (int64_t cy = f0[1]; cy <= f1[1]; ++cy)
            for (int64_t cx = f0[0]; cx <= f1[0]; ++cx) {
                if (hash4(v->seed, cx, cy, cz, 100) % 8 != 0) continue;
                double p[3] = {(double)(cx * kCell) + unit(hash4(v->seed, cx, cy, cz, 101)) * kCell,
                               (double)(cy * kCell) + unit(hash4(v->seed, cx, cy, cz, 102)) * kCell,
                               (double)(cz * kCell) + unit(hash4(v->seed, cx, cy, cz, 103)) * kCell};
                double d[3] = {unit(hash4(v->seed, cx, cy, cz, 104)) - 0.5, unit(hash4(v->seed, cx, cy, cz, 105)) - 0.5,
                               unit(hash4(v->seed, cx, cy, cz, 106)) - 0.5};
                const float val = u16 ? (float)(2500.0 + 1595.0 * unit(hash4(v->seed, cx, cy, cz, 107)))
                                      : (float)(200.0 + 55.0 * unit(hash4(v->seed, cx, cy, cz, 107)));
                for (int s = 0; s < kFibreSteps; ++s) {
                    double e[3];
                    for (int a = 0; a < 3; ++a)
                        e[a] = d[a] + 0.35 * (unit(hash4(v->seed, cx * 131 + s, cy, cz, 200 + (uint64_t)a)) - 0.5);
                    const double nrm = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) + 1e-12;
                    for (int a = 0; a < 3; ++a) p[a] += e[a] / nrm;
                    const int64_t q[3] = {(int64_t)std::llround(p[0]), (int64_t)std::llround(p[1]),
                                          (int64_t)std::llround(p[2])};
                    if (q[0] >= x0 && q[0] < x0 + nx && q[1] >= y0 && q[1] < y0 + ny && q[2] >= z0 && q[2] < z1)
                        acc[(size_t)(((q[2] - z0) * ny + (q[1] - y0)) * nx + (q[0] - x0))] = val;
                }
            }
    // clamp, round, store
    const size_t off = (size_t)((z0 - zbox0) * ny * nx);
    for (size_t i = 0; i < acc.size(); ++i) {
        const double c = std::min(vmax, std::max(0.0, (double)acc[i]));
        const uint32_t u = (uint32_t)std::nearbyint(c);
        if (u16) static_cast<uint16_t *>(dst_box)[off + i] = (uint16_t)u;
        else static_cast<uint8_t *>(dst_box)[off + i] = (uint8_t)u;
    }
}

int pick_threads(int t)
{
    return t > 0 ? t : (int)std::max(1u, std::thread::hardware_concurrency());
}

template <typename F>
void run_threads(int64_t n, int threads, F f)
{
    threads = (int)std::max<int64_t>(1, std::min<int64_t>(threads, n));
    std::atomic<int64_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&] {
            for (int64_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto &x : th) x.join();
}

constexpr int64_t kBase = 256;   // base block edge (a power of two)
constexpr int64_t kTile = 512;   // edge of the tiles that shift it differently

// The base block of (seed, dtype), generated on first use.
const unsigned char *base_block(uint64_t seed, int dtype, int threads)
{
    static std::mutex mu;
    static std::map<std::pair<uint64_t, int>, std::unique_ptr<unsigned char[]>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto &slot = cache[{seed, dtype}];
    if (!slot) {
        const size_t es = dtype == TW_U16 ? 2 : 1;
        slot.reset(new unsigned char[es * (size_t)(kBase * kBase * kBase)]);
        const Gen g{seed, dtype};
        run_threads(kBase / 4, pick_threads(threads), [&](int64_t i) {
            fill_slab(&g, 0, 0, 4 * i, 4 * i + 4, kBase, kBase, slot.get(), 0);
        });
    }
    return slot.get();
}

}  // namespace

extern "C" {

int tw_box_reader_synthetic(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                            void *dst)
{
    const tw_synthetic_volume *v = static_cast<const tw_synthetic_volume *>(user);
    if (!v || !dst || (v->dtype != TW_U8 && v->dtype != TW_U16)) return 1;
    if (x0 < 0 || y0 < 0 || z0 < 0 || nx < 1 || ny < 1 || nz < 1 || x0 + nx > v->sz[0] || y0 + ny > v->sz[1] ||
        z0 + nz > v->sz[2])
        return 2;
    const unsigned char *base = base_block(v->seed, v->dtype, v->threads);
    const int64_t es = v->dtype == TW_U16 ? 2 : 1;
    constexpr int64_t m = kBase - 1;
    run_threads(nz, pick_threads(v->threads), [&](int64_t k) {
        const int64_t z = z0 + k;
        unsigned char *out = static_cast<unsigned char *>(dst) + k * nx * ny * es;
        for (int64_t j = 0; j < ny; ++j) {
            const int64_t y = y0 + j;
            unsigned char *row = out + j * nx * es;
            for (int64_t x = x0; x < x0 + nx;) {
                // the run of this row inside one tile (one shift)
                const int64_t tx = x / kTile, ty = y / kTile, tz = z / kTile;
                const uint64_t h = hash4(v->seed, tx, ty, tz, 999);
                const int64_t sx = (int64_t)(h & m), sy = (int64_t)((h >> 8) & m), sz = (int64_t)((h >> 16) & m);
                const int64_t end = std::min(x0 + nx, (tx + 1) * kTile);
                const unsigned char *brow = base + (((z + sz) & m) * kBase + ((y + sy) & m)) * kBase * es;
                while (x < end) {
                    // contiguous in the base row until it wraps
                    const int64_t bx = (x + sx) & m;
                    const int64_t run = std::min(end - x, kBase - bx);
                    std::memcpy(row + (x - x0) * es, brow + bx * es, (size_t)(run * es));
                    x += run;
                }
            }
        }
    });
    return 0;
}

int tw_box_writer_checksum(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                           const void *src)
{
    tw_checksum *c = static_cast<tw_checksum *>(user);
    if (!c || !src || (c->dtype != TW_U8 && c->dtype != TW_U16)) return 1;
    const bool u16 = c->dtype == TW_U16;
    std::atomic<uint64_t> sum{0}, weighted{0};
    run_threads(nz, pick_threads(c->threads), [&](int64_t k) {
        uint64_t s = 0, w = 0;
        const int64_t z = z0 + k;
        for (int64_t y = 0; y < ny; ++y) {
            const int64_t base = (k * ny + y) * nx;
            for (int64_t x = 0; x < nx; ++x) {
                const uint64_t v = u16 ? static_cast<const uint16_t *>(src)[base + x]
                                       : static_cast<const uint8_t *>(src)[base + x];
                s += v;
                // position-dependent term: a tile delivered to the wrong place changes it
                w += v * (((uint64_t)(x0 + x) * 73856093u) ^ ((uint64_t)(y0 + y) * 19349663u) ^
                          ((uint64_t)z * 83492791u));
            }
        }
        sum += s;
        weighted += w;
    });
    __atomic_add_fetch(&c->sum, sum.load(), __ATOMIC_RELAXED);
    __atomic_add_fetch(&c->weighted, weighted.load(), __ATOMIC_RELAXED);
    __atomic_add_fetch(&c->voxels, (uint64_t)(nx * ny * nz), __ATOMIC_RELAXED);
    return 0;
}

}  // extern "C"
