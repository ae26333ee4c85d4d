// tw_io.cpp -- the reference's file formats at the library boundary: Vaa3D
// raw stacks (.v3draw / .raw), directories of per-Z slice files as a tile
// source, a tile sink that writes finished tiles straight into per-Z slice
// files, and .marker landmark files.
//
// Reference:
//   - raw stack header and payload: loadMetadata_cyf (RawFmtMngr.cpp:332-446)
//     and saveStack2Raw_cyf (Bigwarp.cpp:660-751): the key
//     "raw_image_stack_by_hpeng", one endianness byte ('L' or 'B'), a 2-byte
//     data type code (1, 2 or 4 bytes per voxel), four 4-byte sizes (x, y, z,
//     channels), then the voxels, x fastest, in the file's byte order;
//   - box reads: copyRawFileBlock2Buffer_cyf (RawFmtMngr.cpp:1511-1695) seeks
//     and reads one row at a time; read_2Dtif_BLOCK (Bigwarp.cpp:66-175)
//     reads a box from a directory of slices, one slice per OpenMP thread;
//   - the slice listing: read_2Dtif_dir (dir_make.cpp:175-216), every entry
//     but ".", "..", "mdata.bin" and ".iim.format", sorted by name;
//   - output slices: saveImage_PJ (Bigwarp.cpp:957-1004) names slice z of the
//     stitched output "%07d.raw" with the number z * 10, after a second pass
//     that reassembles the saved tiles (Bigwarp.cpp:229-573).
// Here a box is read with one positioned read per row run (a whole plane
// slab when the box spans full rows), planes in parallel, and the output
// tiles are written into the slice files as they leave the GPU, so no tile
// files and no stitching pass exist.
#include "tw_host.h"

#include <dirent.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace tw;

namespace {

constexpr char kKey[] = "raw_image_stack_by_hpeng";
constexpr int64_t kKeyLen = 24;
constexpr int64_t kHeaderLen = kKeyLen + 1 + 2 + 16;

char host_endian()
{
    const uint32_t a = 0x44332211u;
    unsigned char b[4];
    std::memcpy(b, &a, 4);
    return b[0] == 0x11 ? 'L' : 'B';
}

void swap_bytes(void *p, int64_t n, int es)
{
    unsigned char *c = static_cast<unsigned char *>(p);
    if (es == 2)
        for (int64_t i = 0; i < n; ++i) std::swap(c[2 * i], c[2 * i + 1]);
    else if (es == 4)
        for (int64_t i = 0; i < n; ++i) {
            std::swap(c[4 * i], c[4 * i + 3]);
            std::swap(c[4 * i + 1], c[4 * i + 2]);
        }
}

struct Fd {
    int fd = -1;
    ~Fd() { if (fd >= 0) ::close(fd); }
};

// Reads exactly n bytes at offset off (short reads retried).
bool pread_all(int fd, void *dst, size_t n, int64_t off)
{
    char *p = static_cast<char *>(dst);
    while (n > 0) {
        const ssize_t r = ::pread(fd, p, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return true;
}

bool pwrite_all(int fd, const void *src, size_t n, int64_t off)
{
    const char *p = static_cast<const char *>(src);
    while (n > 0) {
        const ssize_t r = ::pwrite(fd, p, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return true;
}

struct RawHeader {
    int64_t sz[4] = {0, 0, 0, 0};
    int es = 0;        // bytes per voxel (the data type code)
    bool swap = false; // file byte order differs from the host's
};

// Parses the header of an open raw stack; empty string on success.
std::string parse_header(int fd, int64_t file_size, RawHeader &h)
{
    if (file_size < kHeaderLen) return "file too small for a raw stack header";
    unsigned char buf[kHeaderLen];
    if (!pread_all(fd, buf, kHeaderLen, 0)) return "cannot read the header";
    if (std::memcmp(buf, kKey, kKeyLen) != 0) return "unrecognised file format (no raw_image_stack_by_hpeng key)";
    const char e = (char)buf[kKeyLen];
    if (e != 'L' && e != 'B') return "unsupported endianness code in the header";
    h.swap = e != host_endian();
    int16_t code;
    std::memcpy(&code, buf + kKeyLen + 1, 2);
    if (h.swap) swap_bytes(&code, 1, 2);
    if (code != 1 && code != 2 && code != 4) return "unrecognised data type code";
    h.es = code;
    int32_t sz[4];
    std::memcpy(sz, buf + kKeyLen + 3, 16);
    if (h.swap) swap_bytes(sz, 4, 4);
    for (int a = 0; a < 4; ++a) {
        if (sz[a] < 1) return "non-positive size in the header";
        h.sz[a] = sz[a];
    }
    const int64_t payload = h.sz[0] * h.sz[1] * h.sz[2] * h.sz[3] * h.es;
    if (file_size < kHeaderLen + payload) return "file shorter than its header says";
    return std::string();
}

std::string open_raw(const char *path, Fd &f, RawHeader &h)
{
    f.fd = ::open(path, O_RDONLY);
    if (f.fd < 0) return std::string("cannot open ") + path + ": " + std::strerror(errno);
    struct stat st;
    if (::fstat(f.fd, &st) != 0) return std::string("cannot stat ") + path;
    return parse_header(f.fd, (int64_t)st.st_size, h);
}

void make_header(unsigned char out[kHeaderLen], const int64_t sz[4], int es)
{
    std::memcpy(out, kKey, kKeyLen);
    out[kKeyLen] = (unsigned char)host_endian();
    const int16_t code = (int16_t)es;
    std::memcpy(out + kKeyLen + 1, &code, 2);
    int32_t s[4];
    for (int a = 0; a < 4; ++a) s[a] = (int32_t)sz[a];
    std::memcpy(out + kKeyLen + 3, s, 16);
}

int default_threads() { return (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())); }

// Runs f(i) for i in [0, n) on up to `threads` threads; false if any failed.
template <typename F>
bool parallel_for(int64_t n, int threads, F f)
{
    threads = (int)std::max<int64_t>(1, std::min<int64_t>(threads, n));
    if (threads == 1) {
        for (int64_t i = 0; i < n; ++i)
            if (!f(i)) return false;
        return true;
    }
    std::atomic<int64_t> next{0};
    std::atomic<bool> ok{true};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&] {
            for (;;) {
                const int64_t i = next.fetch_add(1);
                if (i >= n || !ok.load()) break;
                if (!f(i)) ok = false;
            }
        });
    for (auto &x : th) x.join();
    return ok.load();
}

// Reads box [x0, x0+nx) x [y0, y0+ny) of plane `plane` (channel-major plane
// index) of an open raw stack into dst (pitch nx): one read for the whole
// row run when the box spans full rows, else one per row.
bool read_plane_box(int fd, const RawHeader &h, int64_t plane, int64_t x0, int64_t y0, int64_t nx, int64_t ny,
                    unsigned char *dst)
{
    const int64_t es = h.es;
    const int64_t row0 = kHeaderLen + ((plane * h.sz[1] + y0) * h.sz[0] + x0) * es;
    if (nx == h.sz[0]) {
        if (!pread_all(fd, dst, (size_t)(nx * ny * es), row0)) return false;
    } else {
        for (int64_t y = 0; y < ny; ++y)
            if (!pread_all(fd, dst + y * nx * es, (size_t)(nx * es), row0 + y * h.sz[0] * es)) return false;
    }
    if (h.swap) swap_bytes(dst, nx * ny, (int)es);
    return true;
}

bool valid_box(const int64_t sz[3], int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz)
{
    return x0 >= 0 && y0 >= 0 && z0 >= 0 && nx > 0 && ny > 0 && nz > 0 && x0 + nx <= sz[0] && y0 + ny <= sz[1] &&
           z0 + nz <= sz[2];
}

int dtype_of(int es) { return es == 1 ? TW_U8 : (es == 2 ? TW_U16 : 0); }

}  // namespace

// ------------------------------------------------------------- slice files

struct tw_slice_dir {
    std::vector<std::string> paths;    // sorted slice files, one per z
    std::vector<RawHeader> heads;
    int64_t sz[3] = {0, 0, 0};
    int es = 0;
    int threads = 1;
};

struct tw_slice_writer {
    std::string dir;
    std::vector<std::string> paths;
    int64_t sz[3] = {0, 0, 0};
    int es = 0;
    int threads = 1;
};

namespace {

std::string slice_name(int64_t z)
{
    char b[32];
    std::snprintf(b, sizeof(b), "%07lld.raw", (long long)(z * 10));
    return b;
}

bool mkdir_p(const std::string &path)
{
    std::string cur;
    size_t i = 0;
    while (i <= path.size()) {
        const size_t j = path.find('/', i);
        cur = path.substr(0, j == std::string::npos ? path.size() : j);
        if (!cur.empty() && ::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
        if (j == std::string::npos) break;
        i = j + 1;
    }
    struct stat st;
    return ::stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

}  // namespace

extern "C" {

tw_status tw_v3draw_read_header(const char *path, int64_t sz[4], int *dtype, int64_t *header_bytes)
{
    if (!path || !sz) return TW_ERR_ARG;
    Fd f;
    RawHeader h;
    if (!open_raw(path, f, h).empty()) return TW_ERR_IO;
    for (int a = 0; a < 4; ++a) sz[a] = h.sz[a];
    if (dtype) *dtype = h.es == 4 ? 4 : dtype_of(h.es);
    if (header_bytes) *header_bytes = kHeaderLen;
    return TW_OK;
}

tw_status tw_v3draw_read(const char *path, void *dst, size_t dst_bytes)
{
    if (!path || !dst) return TW_ERR_ARG;
    Fd f;
    RawHeader h;
    if (!open_raw(path, f, h).empty()) return TW_ERR_IO;
    const int64_t n = h.sz[0] * h.sz[1] * h.sz[2] * h.sz[3];
    if ((size_t)(n * h.es) > dst_bytes) return TW_ERR_ARG;
    const int64_t planes = h.sz[2] * h.sz[3];
    const int64_t plane_b = h.sz[0] * h.sz[1] * h.es;
    unsigned char *d = static_cast<unsigned char *>(dst);
    const bool ok = parallel_for(planes, default_threads(), [&](int64_t p) {
        return read_plane_box(f.fd, h, p, 0, 0, h.sz[0], h.sz[1], d + p * plane_b);
    });
    return ok ? TW_OK : TW_ERR_IO;
}

tw_status tw_v3draw_read_box(const char *path, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny,
                             int64_t nz, void *dst)
{
    if (!path || !dst) return TW_ERR_ARG;
    Fd f;
    RawHeader h;
    if (!open_raw(path, f, h).empty()) return TW_ERR_IO;
    if (!valid_box(h.sz, x0, y0, z0, nx, ny, nz)) return TW_ERR_ARG;
    unsigned char *d = static_cast<unsigned char *>(dst);
    const bool ok = parallel_for(nz, default_threads(), [&](int64_t z) {
        return read_plane_box(f.fd, h, z0 + z, x0, y0, nx, ny, d + z * nx * ny * h.es);
    });
    return ok ? TW_OK : TW_ERR_IO;
}

tw_status tw_v3draw_write(const char *path, const void *data, const int64_t sz[4], int dtype)
{
    if (!path || !data || !sz || (dtype != TW_U8 && dtype != TW_U16)) return TW_ERR_ARG;
    for (int a = 0; a < 4; ++a)
        if (sz[a] < 1 || sz[a] > 0x7fffffff) return TW_ERR_ARG;
    const int es = dtype == TW_U8 ? 1 : 2;
    Fd f;
    f.fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (f.fd < 0) return TW_ERR_IO;
    unsigned char hdr[kHeaderLen];
    make_header(hdr, sz, es);
    if (!pwrite_all(f.fd, hdr, kHeaderLen, 0)) return TW_ERR_IO;
    const int64_t planes = sz[2] * sz[3];
    const int64_t plane_b = sz[0] * sz[1] * es;
    const unsigned char *s = static_cast<const unsigned char *>(data);
    const bool ok = parallel_for(planes, default_threads(), [&](int64_t p) {
        return pwrite_all(f.fd, s + p * plane_b, (size_t)plane_b, kHeaderLen + p * plane_b);
    });
    return ok ? TW_OK : TW_ERR_IO;
}

tw_status tw_slice_dir_open(const char *dir, int threads, tw_slice_dir **out)
{
    if (!dir || !out) return TW_ERR_ARG;
    *out = nullptr;
    DIR *d = ::opendir(dir);
    if (!d) return TW_ERR_IO;
    std::vector<std::string> names;
    while (dirent *e = ::readdir(d)) {
        const std::string n = e->d_name;
        if (n == "." || n == ".." || n == "mdata.bin" || n == ".iim.format") continue;
        names.push_back(n);
    }
    ::closedir(d);
    std::sort(names.begin(), names.end());
    if (names.empty()) return TW_ERR_IO;
    std::unique_ptr<tw_slice_dir> s(new tw_slice_dir);
    s->threads = threads > 0 ? threads : default_threads();
    for (const auto &n : names) {
        const std::string p = std::string(dir) + "/" + n;
        Fd f;
        RawHeader h;
        if (!open_raw(p.c_str(), f, h).empty()) return TW_ERR_IO;
        if (h.sz[2] != 1 || h.sz[3] != 1) return TW_ERR_IO;  // one plane per file
        if (s->heads.empty()) {
            s->sz[0] = h.sz[0];
            s->sz[1] = h.sz[1];
            s->es = h.es;
        } else if (h.sz[0] != s->sz[0] || h.sz[1] != s->sz[1] || h.es != s->es) {
            return TW_ERR_IO;  // slices of one volume share their plane size and type
        }
        s->paths.push_back(p);
        s->heads.push_back(h);
    }
    s->sz[2] = (int64_t)s->paths.size();
    *out = s.release();
    return TW_OK;
}

tw_status tw_slice_dir_info(const tw_slice_dir *d, int64_t sz[3], int *dtype)
{
    if (!d || !sz) return TW_ERR_ARG;
    for (int a = 0; a < 3; ++a) sz[a] = d->sz[a];
    if (dtype) *dtype = dtype_of(d->es);
    return TW_OK;
}

tw_status tw_slice_dir_close(tw_slice_dir *d)
{
    delete d;
    return TW_OK;
}

int tw_box_reader_slices(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                         void *dst)
{
    const tw_slice_dir *s = static_cast<const tw_slice_dir *>(user);
    if (!s || !dst) return 1;
    if (!valid_box(s->sz, x0, y0, z0, nx, ny, nz)) return 2;
    unsigned char *d = static_cast<unsigned char *>(dst);
    const bool ok = parallel_for(nz, s->threads, [&](int64_t z) {
        Fd f;
        f.fd = ::open(s->paths[(size_t)(z0 + z)].c_str(), O_RDONLY);
        if (f.fd < 0) return false;
        return read_plane_box(f.fd, s->heads[(size_t)(z0 + z)], 0, x0, y0, nx, ny, d + z * nx * ny * s->es);
    });
    return ok ? 0 : 3;
}

tw_status tw_slice_writer_create(const char *dir, const int64_t sz[3], int dtype, int threads,
                                 tw_slice_writer **out)
{
    if (!dir || !sz || !out || (dtype != TW_U8 && dtype != TW_U16)) return TW_ERR_ARG;
    *out = nullptr;
    for (int a = 0; a < 3; ++a)
        if (sz[a] < 1 || sz[a] > 0x7fffffff) return TW_ERR_ARG;
    if (!mkdir_p(dir)) return TW_ERR_IO;
    std::unique_ptr<tw_slice_writer> w(new tw_slice_writer);
    w->dir = dir;
    for (int a = 0; a < 3; ++a) w->sz[a] = sz[a];
    w->es = dtype == TW_U8 ? 1 : 2;
    w->threads = threads > 0 ? threads : default_threads();
    // every slice file exists at its final size from the start (header, then
    // zeros), so tiles can be written into it in any order
    const int64_t plane_sz[4] = {sz[0], sz[1], 1, 1};
    unsigned char hdr[kHeaderLen];
    make_header(hdr, plane_sz, w->es);
    const int64_t bytes = kHeaderLen + sz[0] * sz[1] * w->es;
    w->paths.resize((size_t)sz[2]);
    const bool ok = parallel_for(sz[2], w->threads, [&](int64_t z) {
        w->paths[(size_t)z] = std::string(dir) + "/" + slice_name(z);
        Fd f;
        f.fd = ::open(w->paths[(size_t)z].c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (f.fd < 0) return false;
        return pwrite_all(f.fd, hdr, kHeaderLen, 0) && ::ftruncate(f.fd, (off_t)bytes) == 0;
    });
    if (!ok) return TW_ERR_IO;
    *out = w.release();
    return TW_OK;
}

tw_status tw_slice_writer_close(tw_slice_writer *w)
{
    delete w;
    return TW_OK;
}

int tw_box_writer_slices(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                         const void *src)
{
    const tw_slice_writer *w = static_cast<const tw_slice_writer *>(user);
    if (!w || !src) return 1;
    if (!valid_box(w->sz, x0, y0, z0, nx, ny, nz)) return 2;
    const unsigned char *s = static_cast<const unsigned char *>(src);
    const int64_t es = w->es;
    const bool ok = parallel_for(nz, w->threads, [&](int64_t z) {
        Fd f;
        f.fd = ::open(w->paths[(size_t)(z0 + z)].c_str(), O_WRONLY);
        if (f.fd < 0) return false;
        const unsigned char *p = s + z * nx * ny * es;
        const int64_t row0 = kHeaderLen + (y0 * w->sz[0] + x0) * es;
        if (nx == w->sz[0]) return pwrite_all(f.fd, p, (size_t)(nx * ny * es), row0);
        for (int64_t y = 0; y < ny; ++y)
            if (!pwrite_all(f.fd, p + y * nx * es, (size_t)(nx * es), row0 + y * w->sz[0] * es)) return false;
        return true;
    });
    return ok ? 0 : 3;
}

// ------------------------------------------------------------------ markers

tw_status tw_marker_file_read(const char *path, tw_marker *out, int capacity, int *n)
{
    if (!path || !n) return TW_ERR_ARG;
    FILE *f = std::fopen(path, "r");
    if (!f) return TW_ERR_IO;
    std::vector<tw_marker> m;
    char line[4096];
    while (std::fgets(line, sizeof(line), f)) {
        const char *p = line;
        while (*p == ' ' || *p == '\t') ++p;
        if (*p == '#' || *p == '\n' || *p == '\r' || *p == 0) continue;
        // x, y, z are the first three comma-separated fields; the rest
        // (radius, shape, name, comment, colour) is not used by the warp
        double v[3];
        int k = 0;
        const char *q = p;
        while (k < 3) {
            char *end = nullptr;
            v[k] = std::strtod(q, &end);
            if (end == q) break;
            ++k;
            while (*end == ' ' || *end == '\t') ++end;
            if (k < 3) {
                if (*end != ',') break;
                q = end + 1;
            }
        }
        if (k < 3) continue;  // not a marker line
        m.push_back(tw_marker{(float)v[0], (float)v[1], (float)v[2]});
    }
    std::fclose(f);
    *n = (int)m.size();
    if (out) {
        if (capacity < (int)m.size()) return TW_ERR_ARG;
        std::copy(m.begin(), m.end(), out);
    }
    return TW_OK;
}

tw_status tw_marker_file_write(const char *path, const tw_marker *m, int n)
{
    if (!path || (!m && n > 0) || n < 0) return TW_ERR_ARG;
    FILE *f = std::fopen(path, "w");
    if (!f) return TW_ERR_IO;
    std::fprintf(f, "##x,y,z,radius,shape,name,comment, color_r,color_g,color_b\n");
    for (int i = 0; i < n; ++i)
        std::fprintf(f, "%.9g,%.9g,%.9g,0,1,,,255,0,0\n", (double)m[i].x, (double)m[i].y, (double)m[i].z);
    const bool ok = std::fclose(f) == 0;
    return ok ? TW_OK : TW_ERR_IO;
}

}  // extern "C"
