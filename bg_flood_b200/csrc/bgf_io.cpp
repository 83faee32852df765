// Host-side input readers and model set-up helpers: ESRI ASCII grid (.asc)
// bathymetry, the initial block mask and the bed interpolation onto the blocks.
//
// These run once, before the time loop, on the host: they turn a user's files
// into the plain arrays that bgf_set_blocks / bgf_set_bed take.
//
//   bgf_read_asc_head  readbathyASCHead   (src/ReadForcing.cu:2067-2176)
//   bgf_read_asc       readbathyASCzb     (src/ReadForcing.cu:2186-2220)
//   bgf_mask_blocks    CalcInitnblk       (src/Mesh.cu:36-120) / InitBlockxoyo (:257-347)
//   bgf_interp_bathy   interp2BUQ + setedges (src/GridManip.cu:222-330, 380-575)
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/bg_flood_b200.h"
#include "bgf_internal.h"

namespace {

int io_fail(const std::string& msg)
{
    bgf::set_last_error(msg);
    return BGF_EINVAL;
}

bool read_file(const char* path, std::string& out)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, n);
    std::fclose(f);
    return true;
}

// Tokens of `s` separated by `delim`, empty tokens dropped (the reference's split,
// src/ReadInput.cu:1762-1773).
std::vector<std::string> split_skip(const std::string& s, char delim)
{
    std::vector<std::string> out;
    size_t a = 0;
    while (a <= s.size()) {
        size_t b = s.find(delim, a);
        if (b == std::string::npos) b = s.size();
        if (b > a) out.push_back(s.substr(a, b - a));
        a = b + 1;
    }
    return out;
}

// Leading integer / floating value of a header item, as std::stoi / std::stod read
// it (leading blanks skipped, trailing characters ignored); false when none.
bool parse_int(const std::string& s, int& v)
{
    errno = 0;
    char* end = nullptr;
    long r = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || errno) return false;
    v = (int)r;
    return true;
}
bool parse_double(const std::string& s, double& v)
{
    errno = 0;
    char* end = nullptr;
    double r = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) return false;
    v = r;
    return true;
}

double calcres(double dx, int level) { return level < 0 ? dx * (1 << -level) : dx / (1 << level); }

// BilinearInterpolation (src/Util_CPU.cu:129-144) on the four nodes around (x, y),
// (x, y) clamped to the grid; `dyg` is the grid's y spacing.
double bilinear(const bgf_grid& g, double x, double y, double dyg)
{
    const double xi = std::fmax(std::fmin(x, g.xmax), g.xo);
    const double yi = std::fmax(std::fmin(y, g.ymax), g.yo);
    int cfi = (int)std::floor((xi - g.xo) / g.dx);
    cfi = std::min(std::max(cfi, 0), g.nx - 2);
    int cfj = (int)std::floor((yi - g.yo) / dyg);
    cfj = std::min(std::max(cfj, 0), g.ny - 2);
    const int cfip = cfi + 1, cfjp = cfj + 1;
    const double x1 = g.xo + g.dx * cfi, x2 = g.xo + g.dx * cfip;
    const double y1 = g.yo + dyg * cfj, y2 = g.yo + dyg * cfjp;
    const double q11 = g.val[cfi + (size_t)cfj * g.nx], q12 = g.val[cfi + (size_t)cfjp * g.nx];
    const double q21 = g.val[cfip + (size_t)cfj * g.nx], q22 = g.val[cfip + (size_t)cfjp * g.nx];
    const double x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - xi, y2y = y2 - yi, yy1 = yi - y1, xx1 = xi - x1;
    return 1.0 / (x2x1 * y2y1) * (q11 * x2x * y2y + q21 * xx1 * y2y + q12 * x2x * yy1 + q22 * xx1 * yy1);
}

int round_half_away(double v) { return v >= 0 ? (int)(v + 0.5) : (int)(v - 0.5); }

// interp2BUQ (src/GridManip.cu:456-575) in the model precision T: bilinear between
// grid nodes when the cell is not coarser than the grid, else the mean of the grid
// nodes inside the cell, summed in T.
template <class T> T interp_point(const bgf_grid& g, T x, T y, T dx)
{
    if (dx <= (T)g.dx) return (T)bilinear(g, (double)x, (double)y, g.dy);
    const double xmin = x - dx * 0.5, xmax = x + dx * 0.5, ymin = y - dx * 0.5, ymax = y + dx * 0.5;
    const int imin = std::max(round_half_away(std::floor((xmin - g.xo) / g.dx)), 0);
    const int imax = std::min(round_half_away(std::floor((xmax - g.xo) / g.dx)), g.nx - 1);
    const int jmin = std::max(round_half_away(std::floor((ymin - g.yo) / g.dy)), 0);
    const int jmax = std::min(round_half_away(std::floor((ymax - g.yo) / g.dy)), g.ny - 1);
    const int ni = std::max(imax - imin + 1, 1), nj = std::max(jmax - jmin + 1, 1);
    T z = (T)0.0;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++) {
            const int cfi = std::min(imin + i, g.nx - 1), cfj = std::min(jmin + j, g.ny - 1);
            z = z + (T)g.val[cfi + (size_t)cfj * g.nx];
        }
    return z / (T)(ni * nj);
}

template <class T>
void interp_blocks(const bgf_grid& g, int nblk, const int* level, const int* nbr8, const double* bxo,
                   const double* byo, double xo, double yo, double dx0, double* zb)
{
    std::vector<T> t(324);
    for (int ib = 0; ib < nblk; ib++) {
        const double blkdx = calcres(dx0, level ? level[ib] : 0);
        // block origins are held in T by the reference (BlockP<T>::xo)
        const double bx = (double)(T)bxo[ib], by = (double)(T)byo[ib];
        for (int k = 0; k < 324; k++) t[k] = (T)zb[(size_t)ib * 324 + k];
        for (int j = 0; j < 16; j++)
            for (int i = 0; i < 16; i++) {
                const T x = (T)(xo + bx + i * blkdx), y = (T)(yo + by + j * blkdx);
                t[(i + 1) + (j + 1) * 18] = interp_point<T>(g, x, y, (T)blkdx);
            }
        // setedges: the outermost cells on a domain edge take the next cell's value.
        // The left/right test compares the first neighbour twice, as the reference does.
        const int* q = nbr8 + 8 * (size_t)ib;
        auto lr = [&](int A, int B, int ir, int iw) {
            if (A != ib) return;
            const int j0 = 0, j1 = (B == ib) ? 16 : 8;
            for (int j = j0; j < j1; j++) t[(iw + 1) + (j + 1) * 18] = t[(ir + 1) + (j + 1) * 18];
        };
        auto bt = [&](int A, int B, int jr, int jw) {
            if (A != ib && B != ib) return;
            const int i0 = (A == ib) ? 0 : 8, i1 = (B == ib) ? 16 : 8;
            for (int i = i0; i < i1; i++) t[(i + 1) + (jw + 1) * 18] = t[(i + 1) + (jr + 1) * 18];
        };
        lr(q[0], q[1], 1, 0);
        lr(q[2], q[3], 14, 15);
        bt(q[6], q[7], 14, 15);
        bt(q[4], q[5], 1, 0);
        for (int k = 0; k < 324; k++) zb[(size_t)ib * 324 + k] = (double)t[k];
    }
}

bool grid_ok(const bgf_grid* g)
{
    return g && g->val && g->nx >= 2 && g->ny >= 2 && g->dx > 0.0 && g->dy > 0.0;
}

}  // namespace

extern "C" {

int bgf_read_asc_head(const char* path, int* nx, int* ny, double* dx, double* xo, double* yo, double* grdalpha)
{
    if (!path || !nx || !ny || !dx || !xo || !yo) return io_fail("bgf_read_asc_head: null argument");
    std::string text;
    if (!read_file(path, text)) return io_fail(std::string("bathy file could not be opened: ") + path);
    bool pixelreg = true, have_nx = false, have_ny = false, have_dx = false;
    int nxv = 0, nyv = 0;
    double dxv = 0.0, xov = 0.0, yov = 0.0;
    size_t pos = 0;
    int nhead = 0;
    while (nhead < 6) {
        if (pos >= text.size()) return io_fail(std::string("incomplete .asc header (6 lines expected): ") + path);
        size_t e = text.find('\n', pos);
        if (e == std::string::npos) e = text.size();
        const std::string line = text.substr(pos, e - pos);
        pos = e + 1;
        if (line.empty()) continue;  // empty lines do not count
        std::vector<std::string> el = split_skip(line, ' ');
        if (el.size() < 2) el = split_skip(line, '\t');
        if (el.size() < 2) return io_fail("malformed .asc header line: " + line);
        std::string left = el[0];
        while (!left.empty() && left.front() == ' ') left.erase(left.begin());
        while (!left.empty() && left.back() == ' ') left.pop_back();
        const std::string& right = el[1];
        bool ok = true;
        if (left == "ncols") ok = have_nx = parse_int(right, nxv);
        if (left == "nrows") ok = have_ny = parse_int(right, nyv);
        if (left == "cellsize") ok = have_dx = parse_double(right, dxv);
        if (left == "xllcenter") ok = parse_double(right, xov);
        if (left == "yllcenter") {
            pixelreg = false;
            ok = parse_double(right, yov);
        }
        if (left == "xllcorner") {
            pixelreg = false;
            ok = parse_double(right, xov);
        }
        if (left == "yllcorner") ok = parse_double(right, yov);
        if (!ok) return io_fail("unreadable .asc header value: " + line);
        nhead++;
    }
    if (!have_nx || !have_ny || !have_dx || nxv <= 0 || nyv <= 0 || !(dxv > 0.0))
        return io_fail(std::string(".asc header needs ncols, nrows and cellsize: ") + path);
    // The reference treats yllcenter and xllcorner alike: either one shifts both
    // origins by half a cell (src/ReadForcing.cu:2120-2170).
    if (!pixelreg) {
        xov = xov + 0.5 * dxv;
        yov = yov + 0.5 * dxv;
    }
    *nx = nxv;
    *ny = nyv;
    *dx = dxv;
    *xo = xov;
    *yo = yov;
    if (grdalpha) *grdalpha = 0.0;
    return BGF_OK;
}

int bgf_read_asc(const char* path, int nx, int ny, float* val)
{
    if (!path || !val || nx <= 0 || ny <= 0) return io_fail("bgf_read_asc: bad argument");
    std::string text;
    if (!read_file(path, text)) return io_fail(std::string("bathy file could not be opened: ") + path);
    size_t pos = 0;
    for (int k = 0; k < 6; k++) {  // six raw lines, empty ones included
        size_t e = text.find('\n', pos);
        pos = e == std::string::npos ? text.size() : e + 1;
    }
    const char* p = text.c_str() + pos;
    const char* end = text.c_str() + text.size();
    // First file row is the northern one: row jnod = ny-1 down to 0.
    for (int jnod = ny - 1; jnod >= 0; jnod--)
        for (int inod = 0; inod < nx; inod++) {
            while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\v' || *p == '\f')) p++;
            const char c0 = p < end ? *p : 0;
            const char c1 = p + 1 < end ? p[1] : 0;
            const bool numeric = (c0 >= '0' && c0 <= '9') || c0 == '.' ||
                                 ((c0 == '-' || c0 == '+') && ((c1 >= '0' && c1 <= '9') || c1 == '.'));
            if (!numeric)
                return io_fail(std::string(".asc data ends or holds a non-number before ") + std::to_string(nx) + "x" +
                               std::to_string(ny) + " values: " + path);
            char* q = nullptr;
            const float v = std::strtof(p, &q);
            if (q == p) return io_fail(std::string("unreadable .asc value in ") + path);
            val[(size_t)inod + (size_t)jnod * nx] = v;
            p = q;
        }
    return BGF_OK;
}

int bgf_mask_blocks(const bgf_grid* g, int nbx, int nby, double xo, double yo, double levdx, double mask,
                    uint8_t* present, int* nblk)
{
    if (!grid_ok(g) || !present || nbx <= 0 || nby <= 0 || !(levdx > 0.0)) return io_fail("bgf_mask_blocks: bad argument");
    int n = 0;
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            int nmask = 0;
            for (int i = 0; i < 16; i++)
                for (int j = 0; j < 16; j++) {
                    const double x = xo + ((double)i + 16.0 * bx) * levdx + 0.5 * levdx;
                    const double y = yo + ((double)j + 16.0 * by) * levdx + 0.5 * levdx;
                    // this test reads the grid with its x spacing in both directions
                    if (bilinear(*g, x, y, g->dx) >= mask) nmask++;
                }
            const bool keep = nmask < 256;
            present[(size_t)by * nbx + bx] = keep ? 1 : 0;
            n += keep;
        }
    if (nblk) *nblk = n;
    return BGF_OK;
}

int bgf_interp_bathy(const bgf_grid* g, int nblk, const int* level, const int* nbr8, const double* bxo,
                     const double* byo, double xo, double yo, double dx, int doubleprecision, double* zb)
{
    if (!grid_ok(g) || nblk < 0 || !nbr8 || !bxo || !byo || !zb || !(dx > 0.0))
        return io_fail("bgf_interp_bathy: bad argument");
    if (doubleprecision) interp_blocks<double>(*g, nblk, level, nbr8, bxo, byo, xo, yo, dx, zb);
    else interp_blocks<float>(*g, nblk, level, nbr8, bxo, byo, xo, yo, dx, zb);
    return BGF_OK;
}

}  // extern "C"
