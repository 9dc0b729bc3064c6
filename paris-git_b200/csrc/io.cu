// io.cu -- the on-disk formats of the VOF run, fed from the device fields:
// the restart file of backup_VOF_write / backup_VOF_read
// (vofmodules.f90:2033-2085) and the VOF VTK output of output_VOF
// (vofmodules.f90:1908-2031, STRUCTURED_GRID and STRUCTURED_POINTS).
//
// The text follows the Fortran edit descriptors of those routines byte for
// byte: ESw.dEe (scientific, one leading digit, e exponent digits), Ew.d
// (0.ddddd mantissa, two exponent digits or a three-digit exponent without
// the E), Fw.d and Iw, right-justified in their widths.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.cuh"

namespace {

// digits and decimal exponent of |v| rounded to nd significant digits:
// |v| = 0.d1 d2 ... d_nd * 10^e10 (e10 = 0 for v = 0)
void sig_digits(double v, int nd, std::string& digits, int& e10) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*E", nd - 1, std::fabs(v));   // d.dddE+xx, correctly rounded
    digits.clear();
    const char* p = buf;
    for (; *p && *p != 'E'; p++)
        if (*p >= '0' && *p <= '9') digits.push_back(*p);
    const int e = std::atoi(p + 1);
    e10 = v == 0.0 ? 0 : e + 1;
}

void pad_left(std::string& out, const std::string& s, int w) {
    if ((int)s.size() >= w) {
        out += s;
        return;
    }
    out.append(w - s.size(), ' ');
    out += s;
}

// ESw.dEe: [-]d.ddd...E+eee
void fmt_es(std::string& out, double v, int w, int d, int e) {
    std::string dig;
    int e10;
    sig_digits(v, d + 1, dig, e10);
    const int ex = v == 0.0 ? 0 : e10 - 1;
    std::string s;
    if (std::signbit(v)) s += '-';
    s += dig[0];
    s += '.';
    s += dig.substr(1);
    char eb[16];
    std::snprintf(eb, sizeof eb, "E%c%0*d", ex < 0 ? '-' : '+', e, ex < 0 ? -ex : ex);
    s += eb;
    pad_left(out, s, w);
}

// Ew.d: [-]0.ddddE+ee, or [-]0.dddd+eee for |exponent| > 99
void fmt_e(std::string& out, double v, int w, int d) {
    std::string dig;
    int e10;
    sig_digits(v, d, dig, e10);
    std::string s;
    if (std::signbit(v)) s += '-';
    s += "0.";
    s += dig;
    char eb[16];
    const int ae = e10 < 0 ? -e10 : e10;
    if (ae <= 99) std::snprintf(eb, sizeof eb, "E%c%02d", e10 < 0 ? '-' : '+', ae);
    else std::snprintf(eb, sizeof eb, "%c%03d", e10 < 0 ? '-' : '+', ae);
    s += eb;
    pad_left(out, s, w);
}

// Fw.d
void fmt_f(std::string& out, double v, int w, int d) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "%.*f", d, v);
    pad_left(out, buf, w);
}

// Iw
void fmt_i(std::string& out, long v, int w) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%ld", v);
    pad_left(out, buf, w);
}

int download_all(paris_ctx* c, int field, std::vector<double>& h) {
    h.resize(c->L.total);
    return paris_gpu_download(c, field, h.data());
}

int write_text(paris_ctx* c, const char* filename, const std::string& text) {
    FILE* f = std::fopen(filename, "w");
    if (!f) {
        ctx_set_error(c, "cannot open %s for writing: %s", filename, std::strerror(errno));
        return PARIS_BAD_ARGS;
    }
    const size_t n = std::fwrite(text.data(), 1, text.size(), f);
    const int rc = std::fclose(f);
    if (n != text.size() || rc != 0) {
        ctx_set_error(c, "writing %s failed", filename);
        return PARIS_BAD_ARGS;
    }
    return PARIS_OK;
}

// get_flags_and_clip (vofmodules.f90:549-571) on the interior
__global__ void k_flags_clip(double* __restrict__ cv, int8_t* __restrict__ flag, const Layout L, double epsc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const long n = lidx(L, i, blockIdx.y, blockIdx.z);
    const double c = cv[n];
    if (c <= epsc) { flag[n] = 0; cv[n] = 0.0; }
    else if (c >= 1.0 - epsc) { flag[n] = 1; cv[n] = 1.0; }
    else flag[n] = 2;
}

}  // namespace

extern "C" int paris_backup_vof_write(paris_handle_t c, const char* filename, double time, int32_t itimestep) {
    if (!c || !filename) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    std::vector<double> f[5];
    const int fields[5] = {PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_P, PARIS_FIELD_CVOF};
    for (int q = 0; q < 5; q++) PARIS_CHECK(download_all(c, fields[q], f[q]));
    const Layout& L = c->L;
    const int g = L.ng;
    // the previous backup becomes <file>.old (touch + mv of the reference)
    std::string old = std::string(filename) + ".old";
    std::rename(filename, old.c_str());
    std::string s;
    s.reserve((size_t)L.total * 126 + 128);
    // 1100 FORMAT(es17.8e3,7I10): time, itimestep, imin, imax, jmin, jmax, kmin, kmax
    fmt_es(s, time, 17, 8, 3);
    fmt_i(s, itimestep, 10);
    const long lim[6] = {1, L.n[0] + 2L * g, 1, L.n[1] + 2L * g, 1, L.n[2] + 2L * g};
    for (long v : lim) fmt_i(s, v, 10);
    s += '\n';
    // 1200 FORMAT(5es25.16e3) over k, j, i of the whole arrays, ghosts included
    for (long t = 0; t < L.total; t++) {
        for (int q = 0; q < 5; q++) fmt_es(s, f[q][t], 25, 16, 3);
        s += '\n';
    }
    return write_text(c, filename, s);
}

extern "C" int paris_backup_vof_read(paris_handle_t c, const char* filename, double* time, int32_t* itimestep) {
    if (!c || !filename) return PARIS_BAD_ARGS;
    FILE* fp = std::fopen(filename, "r");
    if (!fp) {
        ctx_set_error(c, "cannot open %s: %s", filename, std::strerror(errno));
        return PARIS_BAD_ARGS;
    }
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::string text(sz > 0 ? sz : 0, '\0');
    const size_t got = sz > 0 ? std::fread(&text[0], 1, sz, fp) : 0;
    std::fclose(fp);
    text.resize(got);
    // list-directed read: whitespace-separated values
    const char* p = text.c_str();
    char* end = nullptr;
    auto next = [&](double& out) -> bool {
        out = std::strtod(p, &end);
        if (end == p) return false;
        p = end;
        return true;
    };
    const Layout& L = c->L;
    const int g = L.ng;
    double hdr[8];
    for (int q = 0; q < 8; q++)
        if (!next(hdr[q])) {
            ctx_set_error(c, "backup_read: %s: bad header", filename);
            return PARIS_BAD_ARGS;
        }
    const double want[6] = {1.0, (double)(L.n[0] + 2 * g), 1.0, (double)(L.n[1] + 2 * g), 1.0,
                            (double)(L.n[2] + 2 * g)};
    for (int q = 0; q < 6; q++)
        if (hdr[2 + q] != want[q]) {
            ctx_set_error(c, "Error: backup_read: %s holds another grid", filename);
            return PARIS_BAD_ARGS;
        }
    std::vector<double> f[5];
    for (auto& a : f) a.resize(L.total);
    for (long t = 0; t < L.total; t++)
        for (int q = 0; q < 5; q++)
            if (!next(f[q][t])) {
                ctx_set_error(c, "backup_read: %s: truncated at record %ld", filename, t + 1);
                return PARIS_BAD_ARGS;
            }
    cudaSetDevice(c->dev);
    const int fields[5] = {PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_P, PARIS_FIELD_CVOF};
    for (int q = 0; q < 5; q++) PARIS_CHECK(paris_gpu_upload(c, fields[q], f[q].data()));
    // vof_flag from cvof, then the VOF and velocity ghosts of the restart path
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_VOF_FLAG));
    double* cv = c->fld[PARIS_FIELD_CVOF];
    PARIS_LAUNCH(c, k_flags_clip, dim3(div_up(L.n[0], 128), L.n[1], L.n[2]), 128, 0, cv, c->flag, L, c->d.epsc);
    const long G = ghost_count(L);
    // SetVOFBC + do_all_ghost / do_all_ighost of the restart path (paris.f90:3174-3178)
    PARIS_LAUNCH(c, k_init_ghosts, div_up(G, 256), 256, 0, cv, c->flag, L, c->bnd, ctx_vof_jet(c), G, c->d.epsc);
    for (int q = 0; q < 3; q++) PARIS_CHECK(ctx_ghost_fill(c, c->fld[fields[q]]));
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (time) *time = hdr[0];
    if (itimestep) *itimestep = (int32_t)hdr[1];
    return PARIS_OK;
}

extern "C" int paris_output_vof_vtk(paris_handle_t c, const char* filename, int32_t format, double time,
                                    const int32_t* range, int32_t filtered) {
    if (!c || !filename || (format != PARIS_VTK_STRUCTURED_GRID && format != PARIS_VTK_STRUCTURED_POINTS))
        return PARIS_BAD_ARGS;
    const Layout& L = c->L;
    const int g = L.ng;
    // Fortran indices (1 .. n + 2 ng); default is..ie+1 etc. as the step loop calls it
    int r[6] = {g + 1, g + L.n[0] + 1, g + 1, g + L.n[1] + 1, g + 1, g + L.n[2] + 1};
    if (range)
        for (int q = 0; q < 6; q++) r[q] = range[q];
    for (int a = 0; a < 3; a++) {
        const int lo = r[2 * a], hi = r[2 * a + 1], nt = L.n[a] + 2 * g;
        const int m = filtered ? 1 : 0;   // the filter reads one cell around
        if (lo < 1 + m || hi > nt - m || lo > hi) {
            ctx_set_error(c, "output_VOF: index range %d..%d outside 1..%d", lo, hi, nt);
            return PARIS_BAD_ARGS;
        }
    }
    cudaSetDevice(c->dev);
    std::vector<double> cv;
    PARIS_CHECK(download_all(c, PARIS_FIELD_CVOF, cv));
    const std::vector<double>* X[3] = {&c->h_x, &c->h_y, &c->h_z};
    auto at = [&](int i, int j, int k) {   // Fortran indices
        return cv[(i - 1) + L.pitch * (long)(j - 1) + L.plane * (long)(k - 1)];
    };
    const long np = (long)(r[1] - r[0] + 1) * (r[3] - r[2] + 1) * (r[5] - r[4] + 1);
    std::string s;
    s.reserve(np * (format == PARIS_VTK_STRUCTURED_GRID ? 58 : 15) + 512);
    s += "# vtk DataFile Version 2.0\n";
    s += "grid, time ";
    fmt_f(s, time, 16, 8);
    s += "\nASCII\n";
    if (format == PARIS_VTK_STRUCTURED_POINTS) {
        s += "DATASET STRUCTURED_POINTS\nDIMENSIONS ";
        for (int a = 0; a < 3; a++) fmt_i(s, r[2 * a + 1] - r[2 * a] + 1, 5);
        s += "\nORIGIN ";
        for (int a = 0; a < 3; a++) fmt_f(s, (*X[a])[r[2 * a] - 1], 16, 8);
        s += "\nSPACING ";
        for (int a = 0; a < 3; a++) fmt_f(s, (*X[a])[r[2 * a]] - (*X[a])[r[2 * a] - 1], 16, 8);
        s += '\n';
    } else {
        s += "DATASET STRUCTURED_GRID\nDIMENSIONS ";
        for (int a = 0; a < 3; a++) fmt_i(s, r[2 * a + 1] - r[2 * a] + 1, 5);
        s += "\nPOINTS ";
        fmt_i(s, np, 17);
        s += " double\n";
        for (int k = r[4]; k <= r[5]; k++)
            for (int j = r[2]; j <= r[3]; j++)
                for (int i = r[0]; i <= r[1]; i++) {
                    fmt_e(s, c->h_x[i - 1], 14, 5);
                    fmt_e(s, c->h_y[j - 1], 14, 5);
                    fmt_e(s, c->h_z[k - 1], 14, 5);
                    s += '\n';
                }
    }
    s += "POINT_DATA ";
    fmt_i(s, np, 17);
    s += "\nSCALARS ";
    s += std::string(17, ' ') + "VOF";   // A20 of 'VOF'
    s += " float 1\nLOOKUP_TABLE default\n";
    // output_filtered_VOF weights (vofmodules.f90:142-145)
    const double b1 = 8.0 / 64, b2 = 4.0 / 64, b3 = 2.0 / 64, b4 = 1.0 / 64;
    for (int k = r[4]; k <= r[5]; k++)
        for (int j = r[2]; j <= r[3]; j++)
            for (int i = r[0]; i <= r[1]; i++) {
                double v;
                if (filtered)
                    v = b1 * at(i, j, k) +
                        b2 * (at(i - 1, j, k) + at(i, j - 1, k) + at(i, j, k - 1) + at(i + 1, j, k) + at(i, j + 1, k) +
                              at(i, j, k + 1)) +
                        b3 * (at(i + 1, j + 1, k) + at(i + 1, j - 1, k) + at(i - 1, j + 1, k) + at(i - 1, j - 1, k) +
                              at(i + 1, j, k + 1) + at(i + 1, j, k - 1) + at(i - 1, j, k + 1) + at(i - 1, j, k - 1) +
                              at(i, j + 1, k + 1) + at(i, j + 1, k - 1) + at(i, j - 1, k + 1) + at(i, j - 1, k - 1)) +
                        b4 * (at(i + 1, j + 1, k + 1) + at(i + 1, j + 1, k - 1) + at(i + 1, j - 1, k + 1) +
                              at(i + 1, j - 1, k - 1) + at(i - 1, j + 1, k + 1) + at(i - 1, j + 1, k - 1) +
                              at(i - 1, j - 1, k + 1) + at(i - 1, j - 1, k - 1));
                else
                    v = at(i, j, k);
                fmt_e(s, v, 14, 5);
                s += '\n';
            }
    return write_text(c, filename, s);
}
