// Result files and the hot-start file of the reference, written and read on
// the host (include/ow3d.h, "files"):
//
//  * EP_#####.bin  StoreData (src/IO/StoreData.f90:11-29): a Fortran
//    unformatted sequential file of three records -- (nx, ny) as 32-bit
//    integers, the grid (x, y) and the fields (E, P) as nx*ny doubles each,
//    x fastest, ghost points included. Every record is framed by its length
//    in bytes as a 32-bit integer before and after it (the layout gfortran
//    writes for records below 2 GiB), all little-endian.
//  * fort.NNN      StoreDataAscii (src/IO/StoreDataAscii.f90:21-31): one line
//    "x y E P" per point in the Fortran edit descriptor 4e16.6e3, x fastest,
//    and an empty line after every row of constant y; NNN = 100 + nr.
//  * OceanWave3D.end / OceanWave3D.init  (OceanWave3DTakeATimeStep.f90:146-162,
//    ReadInputFileParameters.f90:113-125, SetupInitialConditions.f90:18-27):
//    a header line, then "Lx Ly Nx Ny time", then "E P" for every interior
//    point, x fastest. The reference writes these lines list-directed; the
//    numbers here carry 17 significant digits, which list-directed input
//    reads back exactly.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ow3d.h"
#include "ow3d_internal.h"

namespace {

thread_local std::string g_io_error;

int fail(const std::string& m) {
    g_io_error = m;
    return OW3D_ERR_BAD_INPUT;
}

std::string join(const char* dir, const std::string& name) {
    if (!dir || !*dir) return name;
    std::string d(dir);
    if (d.back() != '/') d += '/';
    return d + name;
}

bool put_record(FILE* f, const void* a, size_t na, const void* b, size_t nb) {
    const uint64_t len = (uint64_t)na + nb;
    if (len > 0x7fffffffull) return false;
    const int32_t m = (int32_t)len;
    return std::fwrite(&m, 4, 1, f) == 1 && (na == 0 || std::fwrite(a, 1, na, f) == na) &&
           (nb == 0 || std::fwrite(b, 1, nb, f) == nb) && std::fwrite(&m, 4, 1, f) == 1;
}

// One value in the Fortran edit descriptor E16.6E3: a sign, "0.", six digits,
// "E", a signed three-digit exponent, right-justified in 16 columns. The six
// digits are the value correctly rounded to six significant digits.
void fortran_e16_6e3(double v, char* out) {
    char mant[8];
    int e10 = 0;
    bool neg = std::signbit(v) && v != 0.0;
    if (v == 0.0 || !std::isfinite(v)) {
        std::strcpy(mant, "000000");
        e10 = 0;
        if (!std::isfinite(v)) { std::snprintf(out, 17, "%16s", std::isnan(v) ? "NaN" : (neg ? "-Infinity" : "Infinity")); return; }
    } else {
        // d.ddddde+xx with correct rounding, then 0.dddddd E(xx+1)
        char buf[32];
        std::snprintf(buf, sizeof buf, "%.5e", std::fabs(v));
        mant[0] = buf[0];
        std::memcpy(mant + 1, buf + 2, 5);
        mant[6] = 0;
        e10 = std::atoi(buf + 8) + 1;
    }
    char body[24];
    std::snprintf(body, sizeof body, "%s0.%sE%c%03d", neg ? "-" : "", mant, e10 < 0 ? '-' : '+', std::abs(e10));
    std::snprintf(out, 17, "%16s", body);
}

}  // namespace

namespace ow3d {
// One Fortran unformatted sequential record made of `n` parts written back
// to back, framed by its total length as a 32-bit integer (below 2 GiB).
bool write_record(std::FILE* f, const void* const* parts, const size_t* bytes, int n) {
    uint64_t len = 0;
    for (int q = 0; q < n; ++q) len += bytes[q];
    if (len > 0x7fffffffull) return false;
    const int32_t m = (int32_t)len;
    if (std::fwrite(&m, 4, 1, f) != 1) return false;
    for (int q = 0; q < n; ++q)
        if (bytes[q] && std::fwrite(parts[q], 1, bytes[q], f) != bytes[q]) return false;
    return std::fwrite(&m, 4, 1, f) == 1;
}
}  // namespace ow3d

extern "C" {

const char* ow3d_io_last_error(void) { return g_io_error.c_str(); }

int ow3d_write_ep_file(const char* path, int nx, int ny, const double* x, const double* y, const double* E,
                       const double* P) {
    if (!path || nx < 1 || ny < 1 || !x || !y || !E || !P) return fail("ow3d_write_ep_file: bad arguments");
    const size_t n = (size_t)nx * (size_t)ny;
    if (2 * n * sizeof(double) > 0x7fffffffull) return fail("ow3d_write_ep_file: record above 2 GiB");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(std::string("ow3d_write_ep_file: cannot open ") + path + ": " + std::strerror(errno));
    const int32_t dims[2] = {nx, ny};
    bool ok = put_record(f, dims, sizeof dims, nullptr, 0);
    ok = ok && put_record(f, x, n * sizeof(double), y, n * sizeof(double));
    ok = ok && put_record(f, E, n * sizeof(double), P, n * sizeof(double));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? OW3D_OK : fail(std::string("ow3d_write_ep_file: write failed: ") + path);
}

int ow3d_write_ascii_file(const char* path, int nx, int ny, const double* x, const double* y, const double* E,
                          const double* P) {
    if (!path || nx < 1 || ny < 1 || !x || !y || !E || !P) return fail("ow3d_write_ascii_file: bad arguments");
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(std::string("ow3d_write_ascii_file: cannot open ") + path + ": " + std::strerror(errno));
    char a[17], b[17], c[17], d[17];
    bool ok = true;
    for (int j = 0; j < ny && ok; ++j) {
        for (int i = 0; i < nx && ok; ++i) {
            const size_t k = (size_t)j * nx + i;
            fortran_e16_6e3(x[k], a); fortran_e16_6e3(y[k], b); fortran_e16_6e3(E[k], c); fortran_e16_6e3(P[k], d);
            ok = std::fprintf(f, "%s%s%s%s\n", a, b, c, d) > 0;
        }
        ok = ok && std::fputs("\n", f) >= 0;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? OW3D_OK : fail(std::string("ow3d_write_ascii_file: write failed: ") + path);
}

int ow3d_write_end_file(const char* path, double xtank, double ytank, int Nx, int Ny, double time, const double* E,
                        const double* P) {
    if (!path || Nx < 1 || Ny < 1 || !E || !P) return fail("ow3d_write_end_file: bad arguments");
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(std::string("ow3d_write_end_file: cannot open ") + path + ": " + std::strerror(errno));
    bool ok = std::fprintf(f, " Initial conditions outputted from a previous simulation.\n") > 0;
    ok = ok && std::fprintf(f, " %25.17E %25.17E %12d %12d %25.17E\n", xtank, ytank, Nx, Ny, time) > 0;
    const size_t n = (size_t)Nx * (size_t)Ny;
    for (size_t k = 0; k < n && ok; ++k) ok = std::fprintf(f, " %25.17E %25.17E\n", E[k], P[k]) > 0;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? OW3D_OK : fail(std::string("ow3d_write_end_file: write failed: ") + path);
}

int ow3d_read_init_file(const char* path, int Nx, int Ny, double* E, double* P, double* time) {
    if (!path || Nx < 1 || Ny < 1 || !E || !P) return fail("ow3d_read_init_file: bad arguments");
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(std::string("ow3d_read_init_file: cannot open ") + path + ": " + std::strerror(errno));
    // header line (any text)
    int ch;
    while ((ch = std::fgetc(f)) != EOF && ch != '\n') {}
    // list-directed numbers: separators are blanks, commas and new lines; a
    // Fortran exponent may be written with D
    auto next = [&](double& v) -> bool {
        char tok[128];
        int n = 0;
        while ((ch = std::fgetc(f)) != EOF && (ch == ' ' || ch == '\t' || ch == ',' || ch == '\n' || ch == '\r')) {}
        while (ch != EOF && !(ch == ' ' || ch == '\t' || ch == ',' || ch == '\n' || ch == '\r') && n < 127) {
            tok[n++] = (ch == 'd' || ch == 'D') ? 'E' : (char)ch;
            ch = std::fgetc(f);
        }
        tok[n] = 0;
        if (n == 0) return false;
        char* e = nullptr;
        v = std::strtod(tok, &e);
        return e && *e == 0;
    };
    double xt, yt, nx, ny, t0;
    if (!(next(xt) && next(yt) && next(nx) && next(ny) && next(t0))) {
        std::fclose(f);
        return fail("ow3d_read_init_file: second line must hold Lx Ly Nx Ny time");
    }
    if ((int)nx != Nx || (int)ny != Ny) {
        std::fclose(f);
        char m[160];
        std::snprintf(m, sizeof m, "ow3d_read_init_file: the grids must agree (nx=%d, nx IC=%d, ny=%d, ny IC=%d)", Nx,
                      (int)nx, Ny, (int)ny);
        return fail(m);
    }
    const size_t n = (size_t)Nx * (size_t)Ny;
    for (size_t k = 0; k < n; ++k) {
        if (!(next(E[k]) && next(P[k]))) {
            std::fclose(f);
            return fail("ow3d_read_init_file: fewer than Nx*Ny pairs E P");
        }
    }
    std::fclose(f);
    if (time) *time = t0;
    return OW3D_OK;
}

}  // extern "C"
