// snapshot.cuh -- on-disk snapshots and the restart from them.
//
// CAVSNAP1 (src/uniform/snapshot.rs:10-131): magic, nx, ny (u64 LE), then
// rho, ux, uy, T as nx*ny little-endian f64 each, k = iy*nx + ix.
// OCTSNAP1 (src/octree/snapshot.rs:58-170): magic, version u32 = 1, levels
// u32, step u64, n_grids u32, (nx, ny) u64 pairs, then rho, ux, uy, T of each
// grid in the canonical order (L0, hot L1, cold L1[, hot L2, cold L2]).
// Writes are atomic (temporary file in the same directory, then rename), as
// the reference's write_snapshot_atomic.  The restart's bilinear regrid
// (interpolate_field, src/uniform/snapshot.rs:102-131) runs on the device.
#pragma once

#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "solver.cuh"

namespace cav {
namespace snap {

struct Fields {
    int64_t nx = 0, ny = 0;
    std::vector<double> rho, ux, uy, t;
};

struct Oct {
    uint32_t levels = 0;
    uint64_t step = 0;
    std::vector<Fields> grids;
};

inline void put(std::vector<unsigned char>& b, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
}
// The reference writes little-endian fields; so does every CUDA host.
static_assert(sizeof(double) == 8 && sizeof(uint64_t) == 8, "LE 64-bit layout");

inline void write_atomic(const std::string& path, const std::vector<unsigned char>& bytes) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) throw ArgError{CAV_ERR_IO, "snapshot: cannot create " + tmp};
    const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size() && std::fflush(f) == 0 &&
                    fsync(fileno(f)) == 0;
    std::fclose(f);
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw ArgError{CAV_ERR_IO, "snapshot: cannot write " + path};
    }
}

inline std::vector<unsigned char> read_all(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw ArgError{CAV_ERR_IO, "snapshot: cannot open " + path};
    std::vector<unsigned char> d;
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) d.insert(d.end(), buf, buf + n);
    std::fclose(f);
    return d;
}

// write_snapshot_atomic, src/uniform/snapshot.rs:13-61.
inline void write_cavsnap(const std::string& path, int64_t nx, int64_t ny, const double* r, const double* u,
                          const double* v, const double* t) {
    std::vector<unsigned char> b;
    put(b, "CAVSNAP1", 8);
    const uint64_t x = uint64_t(nx), y = uint64_t(ny);
    put(b, &x, 8);
    put(b, &y, 8);
    const size_t n = size_t(nx) * size_t(ny);
    for (const double* a : {r, u, v, t}) put(b, a, n * 8);
    write_atomic(path, b);
}

// read_snapshot, src/uniform/snapshot.rs:64-97.
inline Fields read_cavsnap(const std::string& path) {
    const std::vector<unsigned char> d = read_all(path);
    if (d.size() < 24 || std::memcmp(d.data(), "CAVSNAP1", 8) != 0)
        throw ArgError{CAV_ERR_IO, "snapshot: bad magic or file too short"};
    uint64_t nx, ny;
    std::memcpy(&nx, d.data() + 8, 8);
    std::memcpy(&ny, d.data() + 16, 8);
    if (nx == 0 || ny == 0 || nx > (1u << 20) || ny > (1u << 20))
        throw ArgError{CAV_ERR_IO, "snapshot: implausible grid size"};
    const size_t n = size_t(nx * ny), expect = 24 + 4 * n * 8;
    if (d.size() < expect)
        throw ArgError{CAV_ERR_IO, "snapshot: expected " + std::to_string(expect) + " bytes, read " +
                                       std::to_string(d.size())};
    Fields F;
    F.nx = int64_t(nx);
    F.ny = int64_t(ny);
    size_t off = 24;
    for (std::vector<double>* a : {&F.rho, &F.ux, &F.uy, &F.t}) {
        a->resize(n);
        std::memcpy(a->data(), d.data() + off, n * 8);
        off += n * 8;
    }
    return F;
}

// encode + write_snapshot_atomic, src/octree/snapshot.rs:58-76, 147-165.
inline void write_octsnap(const std::string& path, const Oct& s) {
    std::vector<unsigned char> b;
    put(b, "OCTSNAP1", 8);
    const uint32_t version = 1, ng = uint32_t(s.grids.size());
    put(b, &version, 4);
    put(b, &s.levels, 4);
    put(b, &s.step, 8);
    put(b, &ng, 4);
    for (const Fields& g : s.grids) {
        const uint64_t x = uint64_t(g.nx), y = uint64_t(g.ny);
        put(b, &x, 8);
        put(b, &y, 8);
    }
    for (const Fields& g : s.grids)
        for (const std::vector<double>* a : {&g.rho, &g.ux, &g.uy, &g.t}) put(b, a->data(), a->size() * 8);
    write_atomic(path, b);
}

// decode, src/octree/snapshot.rs:81-142.
inline Oct read_octsnap(const std::string& path) {
    const std::vector<unsigned char> d = read_all(path);
    if (d.size() < 28 || std::memcmp(d.data(), "OCTSNAP1", 8) != 0)
        throw ArgError{CAV_ERR_IO, "octree snapshot: bad magic or file too short"};
    uint32_t version, levels, ng;
    Oct s;
    std::memcpy(&version, d.data() + 8, 4);
    if (version != 1) throw ArgError{CAV_ERR_IO, "octree snapshot: unsupported version " + std::to_string(version)};
    std::memcpy(&levels, d.data() + 12, 4);
    std::memcpy(&s.step, d.data() + 16, 8);
    std::memcpy(&ng, d.data() + 24, 4);
    if (!(levels == 2 || levels == 3) || ng != (levels == 2 ? 3u : 5u))
        throw ArgError{CAV_ERR_IO, "octree snapshot: levels / grid count mismatch"};
    s.levels = levels;
    const size_t dims_end = 28 + size_t(ng) * 16;
    if (d.size() < dims_end) throw ArgError{CAV_ERR_IO, "octree snapshot: truncated header"};
    size_t expect = dims_end;
    s.grids.resize(ng);
    for (uint32_t gi = 0; gi < ng; ++gi) {
        uint64_t nx, ny;
        std::memcpy(&nx, d.data() + 28 + gi * 16, 8);
        std::memcpy(&ny, d.data() + 36 + gi * 16, 8);
        if (nx == 0 || ny == 0 || nx > (1u << 20) || ny > (1u << 20))
            throw ArgError{CAV_ERR_IO, "octree snapshot: implausible grid size"};
        s.grids[gi].nx = int64_t(nx);
        s.grids[gi].ny = int64_t(ny);
        expect += 4 * size_t(nx * ny) * 8;
    }
    if (d.size() != expect)
        throw ArgError{CAV_ERR_IO, "octree snapshot: expected " + std::to_string(expect) + " bytes, read " +
                                       std::to_string(d.size())};
    size_t off = dims_end;
    for (Fields& g : s.grids) {
        const size_t n = size_t(g.nx * g.ny);
        for (std::vector<double>* a : {&g.rho, &g.ux, &g.uy, &g.t}) {
            a->resize(n);
            std::memcpy(a->data(), d.data() + off, n * 8);
            off += n * 8;
        }
    }
    return s;
}

// interpolate_field (src/uniform/snapshot.rs:102-131): bilinear in the
// normalised coordinates of the two grids, in the reference's operation
// order (explicit round-to-nearest operations: no contraction).
static __global__ void k_regrid(const double* __restrict__ src, int nx0, int ny0, double* __restrict__ dst, int nx1,
                                int ny1) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= nx1 || iy >= ny1) return;
    const double vy = ny1 > 1 ? double(iy) / double(ny1 - 1) : 0.0;
    const double sy = __dmul_rn(vy, double(ny0 - 1));
    const int y0 = int(floor(sy));
    const int y1 = y0 + 1 < ny0 - 1 ? y0 + 1 : ny0 - 1;
    const double wy = sy - double(y0);
    const double vx = nx1 > 1 ? double(ix) / double(nx1 - 1) : 0.0;
    const double sx = __dmul_rn(vx, double(nx0 - 1));
    const int x0 = int(floor(sx));
    const int x1 = x0 + 1 < nx0 - 1 ? x0 + 1 : nx0 - 1;
    const double wx = sx - double(x0);
    const double v00 = src[y0 * nx0 + x0], v10 = src[y0 * nx0 + x1];
    const double v01 = src[y1 * nx0 + x0], v11 = src[y1 * nx0 + x1];
    const double a = __dmul_rn(__dmul_rn(v00, 1.0 - wx), 1.0 - wy);
    const double b = __dmul_rn(__dmul_rn(v10, wx), 1.0 - wy);
    const double c = __dmul_rn(__dmul_rn(v01, 1.0 - wx), wy);
    const double e = __dmul_rn(__dmul_rn(v11, wx), wy);
    dst[iy * nx1 + ix] = __dadd_rn(__dadd_rn(__dadd_rn(a, b), c), e);
}

}  // namespace snap
}  // namespace cav
