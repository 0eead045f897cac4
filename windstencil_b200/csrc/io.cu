// io.cu -- the reference's on-disk formats: restart files and metrics files.
//
// Restart file OCFD%08d.dat (OCFD_save / read_file, src/io/OCFD_IO.c:24-226;
// plane records by write_3d / read_3d, src/io/OCFD_IO_mpi.c:563-700), for one
// domain (NX_GLOBAL = nx, ...), little-endian, Fortran-style records:
//   header   int32 12 | int32 Istep | float64 tt | int32 12
//   d, u, v, w, T: per field nz records  int32 nx*ny*8 | nx*ny float64 | int32 nx*ny*8
//                  (plane k, x fastest)
// Metrics file OCFD3d-Jacobi.dat (OCFD_Comput_Jacobian3d.cpp:120-211): no
// header, 13 fields in the same plane records: x, y, z, akx, aky, akz, aix,
// aiy, aiz, asx, asy, asz, ajac.
// Readers check every record marker and the file size; they never guess.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "ws_internal.h"

namespace ws {
namespace {

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

int io_fail(const std::string& what, const char* path) {
    return fail(WS_ERR_IO, what + ": " + (path ? path : "(null)"));
}

bool dims_ok(int nx, int ny, int nz) {
    return nx > 0 && ny > 0 && nz > 0 && (long)nx * ny * 8 < (1L << 31);
}

// one field of nz plane records from dense [nz][ny][nx]
bool write_field(FILE* f, const double* a, int nx, int ny, int nz) {
    const int32_t m = (int32_t)((long)nx * ny * 8);
    const size_t n = (size_t)nx * ny;
    for (int k = 0; k < nz; ++k) {
        if (std::fwrite(&m, 4, 1, f) != 1 || std::fwrite(a + k * n, 8, n, f) != n ||
            std::fwrite(&m, 4, 1, f) != 1)
            return false;
    }
    return true;
}

bool read_field(FILE* f, double* a, int nx, int ny, int nz) {
    const int32_t want = (int32_t)((long)nx * ny * 8);
    const size_t n = (size_t)nx * ny;
    for (int k = 0; k < nz; ++k) {
        int32_t m0 = 0, m1 = 0;
        if (std::fread(&m0, 4, 1, f) != 1 || m0 != want) return false;
        if (std::fread(a + k * n, 8, n, f) != n) return false;
        if (std::fread(&m1, 4, 1, f) != 1 || m1 != want) return false;
    }
    return true;
}

long file_size(FILE* f) {
    if (std::fseek(f, 0, SEEK_END) != 0) return -1;
    const long s = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    return s;
}

long field_bytes(int nx, int ny, int nz) { return ((long)nx * ny * 8 + 8) * nz; }

}  // namespace
}  // namespace ws

using namespace ws;

extern "C" {

int ws_restart_write(const char* path, int nx, int ny, int nz, int32_t istep, double tt,
                     const double* prims) {
    if (!path || !prims || !dims_ok(nx, ny, nz)) return fail(WS_ERR_INVALID, "bad argument");
    File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f) return io_fail("cannot create", path);
    const int32_t m = 12;
    const size_t n = (size_t)nx * ny * nz;
    bool ok = std::fwrite(&m, 4, 1, fh.f) == 1 && std::fwrite(&istep, 4, 1, fh.f) == 1 &&
              std::fwrite(&tt, 8, 1, fh.f) == 1 && std::fwrite(&m, 4, 1, fh.f) == 1;
    for (int q = 0; q < 5 && ok; ++q) ok = write_field(fh.f, prims + q * n, nx, ny, nz);
    if (!ok || std::fflush(fh.f) != 0) return io_fail("write failed", path);
    return WS_OK;
}

int ws_restart_read(const char* path, int nx, int ny, int nz, int32_t* istep, double* tt,
                    double* prims) {
    if (!path || !prims || !istep || !tt || !dims_ok(nx, ny, nz))
        return fail(WS_ERR_INVALID, "bad argument");
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return io_fail("cannot open", path);
    if (file_size(fh.f) != 20 + 5 * field_bytes(nx, ny, nz))
        return io_fail("size does not match a restart file of this grid", path);
    int32_t m0 = 0, m1 = 0;
    if (std::fread(&m0, 4, 1, fh.f) != 1 || m0 != 12 || std::fread(istep, 4, 1, fh.f) != 1 ||
        std::fread(tt, 8, 1, fh.f) != 1 || std::fread(&m1, 4, 1, fh.f) != 1 || m1 != 12)
        return io_fail("bad restart header record", path);
    const size_t n = (size_t)nx * ny * nz;
    for (int q = 0; q < 5; ++q)
        if (!read_field(fh.f, prims + q * n, nx, ny, nz))
            return io_fail("bad plane record", path);
    return WS_OK;
}

int ws_metrics_write(const char* path, int nx, int ny, int nz, const double* fields) {
    if (!path || !fields || !dims_ok(nx, ny, nz)) return fail(WS_ERR_INVALID, "bad argument");
    File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f) return io_fail("cannot create", path);
    const size_t n = (size_t)nx * ny * nz;
    bool ok = true;
    for (int q = 0; q < 13 && ok; ++q) ok = write_field(fh.f, fields + q * n, nx, ny, nz);
    if (!ok || std::fflush(fh.f) != 0) return io_fail("write failed", path);
    return WS_OK;
}

int ws_metrics_read(const char* path, int nx, int ny, int nz, double* fields) {
    if (!path || !fields || !dims_ok(nx, ny, nz)) return fail(WS_ERR_INVALID, "bad argument");
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return io_fail("cannot open", path);
    if (file_size(fh.f) != 13 * field_bytes(nx, ny, nz))
        return io_fail("size does not match a metrics file of this grid", path);
    const size_t n = (size_t)nx * ny * nz;
    for (int q = 0; q < 13; ++q)
        if (!read_field(fh.f, fields + q * n, nx, ny, nz))
            return io_fail("bad plane record", path);
    return WS_OK;
}

}  // extern "C"
