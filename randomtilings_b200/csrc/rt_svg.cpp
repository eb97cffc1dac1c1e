// rt_svg.cpp -- SVG and text output of domains, tilings and dimer covers.
//
// The reference draws with std::ofstream and the stream's default number
// formatting (6 significant digits); these writers produce the same bytes, so
// pictures and matrices written by either side are interchangeable (the tests
// compare SHA-256 digests with the reference's own output).  Each writer cites
// the reference function whose format it keeps.  Output goes through Sink
// (that formatting, written to the file in large blocks), and large pictures
// are formatted by several threads, blocks of rows appended in row order.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/rt_b200.h"
#include "../../include/rt_b200_host.h"
#include "../../include/rt_b200_svg.h"
#include "rt_guard.h"

using rtb::guarded;

namespace {

using Vec = std::vector<int32_t>;
const double kSqrt3 = 1.7320508075688772935274;  // common.h:41

// floor(sqrt(len)), 0 for lengths outside [0, 2^40].
int side_of(int64_t len) {
    if (len < 0 || len > (int64_t)1 << 40) return 0;
    int64_t r = (int64_t)std::llround(std::sqrt((double)len));
    while (r * r > len) --r;
    while ((r + 1) * (r + 1) <= len) ++r;
    return (int)r;
}

// Text output with the number formatting of a default std::ostream -- the
// C++ standard defines `os << double` at the default precision as printf's
// "%.6g" and `os << int` as "%d" -- into a buffer that goes to the file in
// large writes.  Without a file it is a plain buffer (one block of rows).
class Sink {
  public:
    Sink() = default;
    explicit Sink(const char* filename) : f_(std::fopen(filename, "wb")), ok_(f_ != nullptr) {}
    Sink(const Sink&) = delete;
    Sink& operator=(const Sink&) = delete;
    Sink(Sink&&) = default;
    ~Sink() { close(); }

    Sink& operator<<(const char* s) {
        buf_.append(s);
        return spill();
    }
    Sink& operator<<(const std::string& s) {
        buf_.append(s);
        return spill();
    }
    template <class T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    Sink& operator<<(T v) {
        char tmp[24];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v);
        buf_.append(tmp, r.ptr);
        return spill();
    }
    Sink& operator<<(double x) {
        put_double(x);
        return spill();
    }
    void append(const Sink& o) {
        buf_.append(o.buf_);
        spill();
    }
    void clear() { buf_.clear(); }
    // Flushes and closes the file; false if it could not be opened or written.
    bool close() {
        if (f_) {
            if (!buf_.empty() && std::fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) ok_ = false;
            buf_.clear();
            if (std::fclose(f_) != 0) ok_ = false;
            f_ = nullptr;
        }
        return ok_;
    }

  private:
    Sink& spill() {
        if (f_ && buf_.size() >= (1u << 22)) {
            if (std::fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) ok_ = false;
            buf_.clear();
        }
        return *this;
    }
    // "%.6g".  Exact multiples of 1/2 below 1e5 in magnitude -- every
    // coordinate of the lattice pictures -- have at most six significant
    // digits, which %.6g prints in full: the integer part, then ".5" for an
    // odd half.  Anything else (and -0) goes through snprintf.
    void put_double(double x) {
        const double a = std::fabs(x), t = 2 * a;
        if (a < 1e5 && t == std::floor(t) && !(x == 0 && std::signbit(x))) {
            const int64_t k = (int64_t)t;
            if (x < 0) buf_.push_back('-');
            char tmp[24];
            const auto r = std::to_chars(tmp, tmp + sizeof tmp, k >> 1);
            buf_.append(tmp, r.ptr);
            if (k & 1) buf_.append(".5");
            return;
        }
        char tmp[48];
        const int len = std::snprintf(tmp, sizeof tmp, "%.6g", x);
        buf_.append(tmp, (size_t)std::max(0, len));
    }

    std::FILE* f_ = nullptr;
    bool ok_ = true;
    std::string buf_;
};

// Threads formatting rows: RT_WRITER_THREADS if set, else the host's cores (at most 64).
unsigned writer_threads() {
    if (const char* e = std::getenv("RT_WRITER_THREADS")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v >= 1) return (unsigned)std::min(v, 256L);
    }
    return std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
}

// row(s, i) writes row i (lo <= i < hi) to s.  Small pictures are written in
// order on this thread; large ones in windows of consecutive row blocks,
// one block per thread, each into its own buffer, appended in row order --
// the same bytes as the sequential loop, whatever the thread count.
template <class F>
void for_rows(Sink& o, int lo, int hi, int64_t cells_per_row, const F& row) {
    const int64_t rows = (int64_t)hi - lo;
    const unsigned T = writer_threads();
    if (rows <= 0) return;
    if (T <= 1 || rows * std::max<int64_t>(1, cells_per_row) < (1 << 16)) {
        for (int i = lo; i < hi; ++i) row(o, i);
        return;
    }
    const int64_t blk = std::max<int64_t>(1, (1 << 15) / std::max<int64_t>(1, cells_per_row));
    std::vector<Sink> part(T);
    for (int64_t w0 = lo; w0 < hi; w0 += blk * T) {
        std::vector<std::thread> th;
        for (unsigned k = 0; k < T; ++k) {
            const int64_t a = w0 + (int64_t)k * blk, b = std::min<int64_t>(hi, a + blk);
            if (a >= b) break;
            part[k].clear();
            th.emplace_back([&row, &part, k, a, b] {
                for (int64_t i = a; i < b; ++i) row(part[k], (int)i);
            });
        }
        for (size_t k = 0; k < th.size(); ++k) {
            th[k].join();
            o.append(part[k]);
        }
    }
}

const char* kSvgOpen = "<svg xmlns='http://www.w3.org/2000/svg' xmlns:xlink=\"http://www.w3.org/1999/xlink\" ";

// <use xlink:href = "#id" x = "X" y = "Y"/>  (the spaced form) or without spaces.
void use(Sink& o, const char* id, double x, double y, bool spaced) {
    if (spaced)
        o << "<use xlink:href = \"#" << id << "\" x = \"" << x << "\" y = \"" << y << "\"/>\n";
    else
        o << "<use xlink:href=\"#" << id << "\" x=\"" << x << "\" y=\"" << y << "\"/>\n";
}

// Header of the triangular-lattice pictures (viewBox 1.5 M, aspect 433.013:500).
void tri_header(Sink& o, double m) {
    o << kSvgOpen << "height=\"433.013\" width=\"500\" viewBox=\"0 0 " << 3 / 2.0 * m << " " << 3 / 2.0 * m
      << "\" preserveAspectRatio=\"none\">\n";
}

rt_status finish(Sink& f) { return f.close() ? RT_OK : RT_E_INVAL; }

// ---- rectangle-triangle face pictures (RectTriangleTiler.cpp:567-697) ----------
double vx(int i, int j) { return 20 * (i * 1 / 2.0 + j); }
double vy(int i, int) { return 20 * (i * kSqrt3 / 2.0); }

void face_picture(Sink& o, int type, int i, int j) {
    static const char* kFill[4] = {
        "", "\" style=\"fill:midnightblue;stroke:midnightblue;stroke-width:.4\" />\n",
        "\" style=\"fill:slategrey;stroke:slategrey;stroke-width:.4\" />\n",
        "\" style=\"fill:lightsteelblue;stroke:lightsteelblue;stroke-width:.4\" />\n"};
    const char* edge = " style=\"stroke:rgb(0,0,0);stroke-width:.5\" stroke-linecap = \"round\" />\n";
    // Corners P, Q, R of the face and the midpoints p, q, r of the opposite
    // sides; per face type: which corner polygons / edges / half-edges are drawn.
    bool PQ = false, PR = false, QR = false, p = false, q = false, r = false;
    int whole = 0, pPR = 0, pPQ = 0, rRQ = 0, rRP = 0, qQR = 0, qQP = 0;
    switch (type) {
        case 1: PR = QR = r = true, whole = 1; break;
        case 2: QR = PQ = q = true, whole = 3; break;
        case 3: PQ = PR = p = true, whole = 2; break;
        case 4: r = true, whole = 2; break;
        case 5: q = true, whole = 1; break;
        case 6: p = true, whole = 3; break;
        case 7: PQ = true, whole = 2; break;
        case 8: PR = true, whole = 1; break;
        case 9: QR = true, whole = 3; break;
        case 10: rRP = 1, rRQ = 2, r = PR = true; break;
        case 11: qQP = 1, qQR = 3, q = QR = true; break;
        case 12: pPQ = 2, pPR = 3, p = PQ = true; break;
        case 13: rRP = 2, rRQ = 1, r = QR = true; break;
        case 14: qQP = 3, qQR = 1, q = PQ = true; break;
        case 15: pPQ = 3, pPR = 2, p = PR = true; break;
        default: break;
    }
    double Px, Py, Qx, Qy, Rx, Ry;
    if (j % 2 == 1) {
        Px = vx(i + 1, j / 2), Py = vy(i + 1, j / 2);
        Qx = vx(i + 1, j / 2 + 1), Qy = vy(i + 1, j / 2 + 1);
        Rx = vx(i, j / 2 + 1), Ry = vy(i, j / 2 + 2);
    } else {
        Px = vx(i, j / 2 + 1), Py = vy(i, j / 2 + 1);
        Qx = vx(i, j / 2), Qy = vy(i, j / 2);
        Rx = vx(i + 1, j / 2), Ry = vy(i + 1, j / 2);
    }
    const double px = (Rx + Qx) / 2, py = (Ry + Qy) / 2;
    const double qx = (Px + Rx) / 2, qy = (Py + Ry) / 2;
    const double rx = (Px + Qx) / 2, ry = (Py + Qy) / 2;
    auto poly = [&](double ax, double ay, double bx, double by, double cx, double cy, int colour) {
        o << "<polygon points=\"" << ax << "," << ay << " " << bx << "," << by << " " << cx << "," << cy << " "
          << kFill[colour];
    };
    auto line = [&](double ax, double ay, double bx, double by) {
        o << "<line x1=\"" << ax << "\" y1=\"" << ay << "\" x2=\"" << bx << "\" y2=\"" << by << "\"" << edge;
    };
    if (whole > 0) poly(Px, Py, Qx, Qy, Rx, Ry, whole);
    if (pPR > 0) poly(Px, Py, px, py, Rx, Ry, pPR);
    if (pPQ > 0) poly(Px, Py, px, py, Qx, Qy, pPQ);
    if (rRQ > 0) poly(Rx, Ry, rx, ry, Qx, Qy, rRQ);
    if (rRP > 0) poly(Rx, Ry, rx, ry, Px, Py, rRP);
    if (qQR > 0) poly(Qx, Qy, qx, qy, Rx, Ry, qQR);
    if (qQP > 0) poly(Qx, Qy, qx, qy, Px, Py, qQP);
    if (PQ) line(Px, Py, Qx, Qy);
    if (PR) line(Px, Py, Rx, Ry);
    if (QR) line(Rx, Ry, Qx, Qy);
    if (p) line(Px, Py, px, py);
    if (q) line(Qx, Qy, qx, qy);
    if (r) line(Rx, Ry, rx, ry);
}

}  // namespace

extern "C" {

// ---- dominoes ------------------------------------------------------------------
rt_status rt_domino_domain_svg(const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!d || !filename) return RT_E_INVAL;
        const int m = side_of(dlen);
        Sink o(filename);
        o << kSvgOpen << "height=\"500\" width=\"500\" viewBox=\"0 0 " << m << " " << m << "\">\n";
        o << "<defs>\n";
        o << "<g id=\"b\">  <polygon points = \"-.5,-.5 .5,-.5 .5,.5 -.5,.5\" fill=\"blue\"/> </g>\n";
        o << "<g id=\"w\">  <polygon points = \"-.5,-.5 .5,-.5 .5,.5 -.5,.5\" fill=\"grey\"/> </g>\n";
        o << "</defs>\n";
        for_rows(o, 0, m, m, [&](Sink& row_out, int i) {
            for (int j = 0; j < m; ++j)
                if (d[(size_t)i * m + j] == 1) use(row_out, (i + j) % 2 == 0 ? "b" : "w", j + .5, i + .5, true);
        });
        o << "</svg>";
        return finish(o);
    });
}

// Dominoes as rectangles anchored at the vertex whose up (1) / left-edge (4)
// bit is set (DominoTiler::TilingToSVG, DominoTiler.cpp:613-640) or as pairs
// of discs (MayaToSVG, :642-681).
static rt_status domino_pairs_svg(const int32_t* t, int64_t tlen, const char* filename, bool maya) {
    if (!t || !filename) return RT_E_INVAL;
    const int n = side_of(tlen);
    Sink o(filename);
    o << kSvgOpen << "height=\"500\" width=\"500\" viewBox=\"0 0 " << (n - 1) << " " << (n - 1) << "\">\n";
    o << "<defs>\n";
    if (!maya) {
        const char* h = "<polygon points = \"-1,0 -1,-1 1,-1 1,0\" fill=\"white\" stroke=\"black\" stroke-width=\".05\"/>";
        const char* v = "<polygon points = \"-1,-1 0,-1 0,1 -1,1\" fill=\"white\" stroke=\"black\" stroke-width=\".05\"/>";
        o << "<g id=\"h1\">  " << h << " </g>\n";
        o << "<g id=\"v1\">  " << v << " </g>\n";
        o << "<g id=\"h2\">  " << h << " </g>\n";
        o << "<g id=\"v2\">  " << v << " </g>\n";
    } else {
        auto disc = [&](const char* cx, const char* cy, const char* fill) {
            o << "<circle cx=\"" << cx << "\" cy=\"" << cy << "\" r=\".4\" stroke=\"black\" stroke-width=\".02\" fill=\""
              << fill << "\"/>";
        };
        const char* names[4] = {"h1", "h2", "v1", "v2"};
        for (int g = 0; g < 4; ++g) {
            const char* fill = g % 2 == 0 ? "black" : "white";
            o << "<g id=\"" << names[g] << "\">";
            if (g < 2) {
                disc("-.5", "-.5", fill);
                o << " ";
                disc(".5", "-.5", fill);
            } else {
                disc("-.5", "-.5", fill);
                o << " ";
                disc("-.5", ".5", fill);
            }
            o << "</g>\n";
        }
    }
    o << "</defs>\n";
    for_rows(o, 0, n, n, [&](Sink& row_out, int i) {
        for (int j = 0; j < n; ++j) {
            const int32_t v = t[(size_t)i * n + j];
            const bool odd = (i + j) % 2 == 1;
            if ((v & 1) == 1) use(row_out, odd ? "h1" : "h2", j, i, true);
            if ((v & 4) == 4) use(row_out, odd ? "v1" : "v2", j, i, true);
        }
    });
    o << "</svg>";
    return finish(o);
}

rt_status rt_domino_tiling_svg(const int32_t* t, int64_t tlen, const char* filename) {
    return guarded([&]() -> rt_status {
        return domino_pairs_svg(t, tlen, filename, false);
    });
}

rt_status rt_domino_maya_svg(const int32_t* t, int64_t tlen, const char* filename) {
    return guarded([&]() -> rt_status {
        return domino_pairs_svg(t, tlen, filename, true);
    });
}

// DominoTiler::DimerToSVG(t, d) (DominoTiler.cpp:538-611); d = NULL takes the
// domain from the tiling (DimerToSVG(t), :533-536).
rt_status rt_domino_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen), m = n - 1;
        Vec dom;
        if (!d) {
            dom.assign((size_t)m * m, 0);
            for (int i = 0; i < m; ++i)
                for (int j = 0; j < m; ++j)
                    if ((t[(size_t)i * n + j] & (2 + 8)) || (t[(size_t)(i + 1) * n + j + 1] & (1 + 4))) dom[(size_t)i * m + j] = 1;
            d = dom.data();
            dlen = (int64_t)dom.size();
        }
        if (dlen < (int64_t)m * m) return RT_E_INVAL;
        // The reference indexes d[i M + j +- 1] and d[(i +- 1) M + j] as flat
        // offsets (DominoTiler.cpp:571-592): a column step past the edge reads
        // the next row's first cell, and the row after the last one lies past
        // the array.  The same flat reads here, with offsets past the array
        // reading as empty (the builders' padded domains never reach them).
        auto D = [&](int i, int j) {
            const int64_t k = (int64_t)i * m + j;
            return k >= 0 && k < (int64_t)m * m ? d[k] : 0;
        };
        Sink o(filename);
        o << kSvgOpen << "height=\"500\" width=\"500\" viewBox=\"0 0 " << m << " " << m << "\">\n";
        o << "<defs>\n";
        o << "<g id=\"hd\">  <polyline points= \"-.5,0 .5,0\" stroke=\"red\" stroke-width=\".05\"/> </g>\n";
        o << "<g id=\"he\">  <polyline points= \"-.5,0 .5,0\" stroke=\"black\" stroke-width=\".01\"/> </g>\n";
        o << "<g id=\"vd\">  <polyline points= \"0,-.5 0,.5\" stroke=\"red\" stroke-width=\".05\"/> </g>\n";
        o << "<g id=\"ve\">  <polyline points= \"0,-.5 0,.5\" stroke=\"black\" stroke-width=\".01\"/> </g>\n";
        o << "<g id=\"b\">  <circle cx=\"0\" cy=\"0\" r=\".1\" stroke=\"black\" stroke-width=\".02\" fill=\"black\"/> </g> \n";
        o << "<g id=\"w\">  <circle cx=\"0\" cy=\"0\" r=\".1\" stroke=\"black\" stroke-width=\".02\" fill=\"white\" /> </g>\n";
        o << "</defs>\n";
        for_rows(o, 0, n, n, [&](Sink& row_out, int i) {
            for (int j = 0; j < n; ++j) {
                const double x = j, y = i;
                const int32_t v = t[(size_t)i * n + j];
                if ((v & 1) == 1) use(row_out, "hd", x, y - .5, false);
                if ((v & 4) == 4) use(row_out, "vd", x - .5, y, false);
            }
        });
        for_rows(o, 1, m, m, [&](Sink& row_out, int i) {
            for (int j = 1; j < m; ++j) {
                if (D(i, j) != 1) continue;
                const double x = j + .5, y = i + .5;
                if ((i + j) % 2 == 1) {
                    if (D(i, j + 1) == 1) use(row_out, "he", x + .5, y, false);
                    if (D(i, j - 1) == 1) use(row_out, "he", x - .5, y, false);
                }
                if (D(i - 1, j) == 1) use(row_out, "ve", x, y - .5, false);
                if (D(i + 1, j) == 1) use(row_out, "ve", x, y + .5, false);
            }
        });
        for_rows(o, 1, m, m, [&](Sink& row_out, int i) {
            for (int j = 1; j < m; ++j)
                if (D(i, j) == 1) use(row_out, (i + j) % 2 == 0 ? "b" : "w", j + .5, i + .5, true);
        });
        o << "</svg>";
        return finish(o);
    });
}

// ---- lozenges ----------------------------------------------------------------------
// LozengeTiler::DomainToSVG (LozengeTiler.cpp:593-613).
rt_status rt_lozenge_domain_svg(const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!d || !filename) return RT_E_INVAL;
        const int m = side_of(dlen / 2);
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"w\">  <polygon points = \"0,1 .5,0 1,1\" fill=\"lightsteelblue\"/> </g>\n";
        o << "<g id=\"b\">  <polygon points = \"0,0 1,0 .5,1\" fill=\"slategrey\"/> </g>\n";
        o << "</defs>\n";
        for_rows(o, 0, m, 2 * m, [&](Sink& row_out, int i) {
            for (int j = 0; j < 2 * m; ++j)
                if (d[(size_t)i * 2 * m + j] == 1) use(row_out, j % 2 == 0 ? "b" : "w", .5 * j + .5 * i, i, true);
        });
        o << "</svg>";
        return finish(o);
    });
}

// LozengeTiler::TilingToSVG (LozengeTiler.cpp:565-590).
rt_status rt_lozenge_tiling_svg(const int32_t* t, int64_t tlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen), m = n - 1;
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"r\">  <polygon points = \"0,0 -1,0 -.5,-1 .5,-1\" fill=\"midnightblue\"/> </g>\n";
        o << "<g id=\"g\">  <polygon points = \"0,0 1,0 .5,-1 -.5,-1\" fill=\"lightsteelblue\"/> </g>\n";
        o << "<g id=\"b\">  <polygon points = \"0,0 .5,-1 1,0 .5,1\" fill=\"slategrey\"/> </g>\n";
        o << "</defs>\n";
        for_rows(o, 1, n - 1, n, [&](Sink& row_out, int i) {
            for (int j = 1; j < n - 1; ++j) {
                const int32_t v = t[(size_t)i * n + j];
                if ((v & 1) == 1) use(row_out, "r", j + .5 * i, i, true);
                if ((v & 2) == 2) use(row_out, "g", j + .5 * i, i, true);
                if ((v & 8) == 8) use(row_out, "b", j + .5 * i, i, true);
            }
        });
        o << "</svg>";
        return finish(o);
    });
}

// LozengeTiler::DimerToSVG(t, d) (LozengeTiler.cpp:487-562); d = NULL takes
// the domain from the tiling (TilingToDomain, :436-462).
rt_status rt_lozenge_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen), m = n - 1;
        Vec dom;
        if (!d) {
            dom.assign((size_t)2 * m * m, 0);
            auto set = [&](int r, int c) {
                if (r >= 0 && r < m && c >= 0 && c < 2 * m) dom[(size_t)r * 2 * m + c] = 1;
            };
            for (int i = 0; i < n - 1; ++i)
                for (int j = 0; j < n - 1; ++j) {
                    const int32_t v = t[(size_t)i * n + j];
                    if (v & 1) set(i - 1, 2 * j), set(i - 1, 2 * j - 1);
                    if (v & 2) set(i - 1, 2 * j), set(i - 1, 2 * j + 1);
                    if (v & 8) set(i - 1, 2 * j + 1), set(i, 2 * j);
                }
            d = dom.data();
            dlen = (int64_t)dom.size();
        }
        if (dlen < (int64_t)2 * m * m + 2 * m) {  // the reference reads row N-1 (one past the domain)
            Vec pad(d, d + dlen);
            pad.resize((size_t)2 * m * (m + 2), 0);
            dom.swap(pad);
            d = dom.data();
        }
        auto D = [&](int i, int j) { return d[(size_t)i * m * 2 + j]; };
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"e1\">  <polyline points= \"-.5,-.33333333333 0,-.666666666666\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"e2\">  <polyline points= \"0,-.666666666 .5,-.333333333333\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"e8\">  <polyline points= \".5,-.333333333333 .5,.333333333333\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"d1\">  <polyline points= \"-.5,-.33333333333 0,-.666666666666\" stroke=\"black\" stroke-width=\".025\"/> </g>\n";
        o << "<g id=\"d2\">  <polyline points= \"0,-.666666666 .5,-.333333333333\" stroke=\"black\" stroke-width=\".025\"/> </g>\n";
        o << "<g id=\"d8\">  <polyline points= \".5,-.333333333333 .5,.333333333333\" stroke=\"black\" stroke-width=\".025\"/> </g>\n";
        o << "<g id=\"b\">  <ellipse cx=\".5\" cy=\".333333333333\" rx=\".1\" ry=\".11547\" stroke=\"black\" stroke-width=\".02\" fill=\"black\"/> </g> \n";
        o << "<g id=\"w\">  <ellipse cx=\".5\" cy=\".666666666666\" rx=\".1\"  ry=\".11547\" stroke=\"black\" stroke-width=\".02\" fill=\"white\" /> </g>\n";
        o << "</defs>\n";
        for_rows(o, 1, n - 1, n, [&](Sink& row_out, int i) {
            for (int j = 1; j < n - 1; ++j) {
                const int32_t v = t[(size_t)i * n + j];
                if ((v & 1) == 1) use(row_out, "d1", j + .5 * i, i, true);
                if ((v & 2) == 2) use(row_out, "d2", j + .5 * i, i, true);
                if ((v & 8) == 8) use(row_out, "d8", j + .5 * i, i, true);
            }
        });
        for_rows(o, 1, n - 1, 2 * n, [&](Sink& row_out, int i) {
            for (int j = 1; j < 2 * n - 1; ++j)
                if (D(i, j) == 1 && j % 2 == 0) {
                    if (D(i, j - 1) == 1) use(row_out, "e1", .5 + .5 * j + .5 * i, i + 1, true);
                    if (D(i, j + 1) == 1) use(row_out, "e2", .5 + .5 * j + .5 * i, i + 1, true);
                    if (D(i + 1, j - 1) == 1) use(row_out, "e8", .5 + .5 * j + .5 * i, i + 1, true);
                }
        });
        for_rows(o, 1, n - 1, 2 * n, [&](Sink& row_out, int i) {
            for (int j = 1; j < 2 * n - 1; ++j)
                if (D(i, j) == 1) use(row_out, j % 2 == 0 ? "b" : "w", .5 * i + .5 * j, i, true);
        });
        o << "</svg>";
        return finish(o);
    });
}

// LozengeTiler::PrintDomain (LozengeTiler.cpp:391-403): the M x 2M domain as text.
rt_status rt_lozenge_print_domain(const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!d || !filename) return RT_E_INVAL;
        const int m = side_of(dlen / 2);
        Sink o(filename);
        for_rows(o, 0, m, 2 * m, [&](Sink& row_out, int i) {
            for (int j = 0; j < 2 * m; ++j) row_out << d[(size_t)i * 2 * m + j] << " ";
            row_out << "\n";
        });
        return finish(o);
    });
}

// ---- rectangle-triangle (RectTriangleTiler::TilingToSVG, :567-592) -------------------
rt_status rt_recttri_tiling_svg(const int32_t* t, int64_t tlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen), m = n - 1;
        const double W = kSqrt3 * 2 * (n + 1), H = 3 / 2.0 * (n + 1), s = 20;
        Sink o(filename);
        o << "<svg xmlns='http://www.w3.org/2000/svg' height=\"" << s * H << "\" width=\"" << s * W << "\" >\n";
        for_rows(o, 0, m, 8 * m, [&](Sink& row_out, int i) {
            for (int j = 0; j < m; ++j) {
                face_picture(row_out, (t[(size_t)i * n + j + 1] & (0xf << 4)) >> 4, i, 2 * j + 1);
                face_picture(row_out, t[(size_t)i * n + j] & 0xf, i, 2 * j);
            }
        });
        o << "</svg>";
        return finish(o);
    });
}

// ---- triangular-lattice dimers (TriangleDimerTiler.cpp:772-902) ------------------------
rt_status rt_tridimer_domain_svg(const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!d || !filename) return RT_E_INVAL;
        const int m = side_of(dlen / 2);
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"w\">  <polygon points = \"0,1 .5,0 1,1\" fill=\"paleturquoise\"/> </g>\n";
        o << "<g id=\"b\">  <polygon points = \"0,0 1,0 .5,1\" fill=\"deepskyblue\"/> </g>\n";
        o << "</defs>\n";
        for_rows(o, 0, m, 2 * m, [&](Sink& row_out, int i) {
            for (int j = 0; j < 2 * m; ++j)
                if (d[(size_t)i * m * 2 + j] == 1) use(row_out, j % 2 == 0 ? "b" : "w", .5 * j + .5 * i, i, true);
        });
        o << "</svg>";
        return finish(o);
    });
}

rt_status rt_tridimer_tiling_svg(const int32_t* t, int64_t tlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen), m = n / 2;
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"dR\">  <polygon points = \"1,-0.6666666667 0.5,-0.3333333333 0.5,0.3333333333 0,0.6666666667 0,1.333333333 0.5,1.666666667 1,1.333333333 1,0.6666666667 1.5,0.3333333333 1.5,-0.3333333333\" fill=\"midnightblue\" stroke=\"black\" stroke-width=\".05\"/></g>\n";
        o << "<g id=\"dL\">  <polygon points = \"0,-0.6666666667 0.5,-0.3333333333 0.5,0.3333333333 1,0.6666666667 1,1.333333333 0.5,1.666666667 0,1.333333333 0,0.6666666667 -0.5,0.3333333333 -0.5,-0.3333333333\" fill=\"lightsteelblue\" stroke=\"black\" stroke-width=\".05\"/></g>\n";
        o << "<g id=\"dH\">  <polygon points = \"0,-0.6666666667 0.5,-0.3333333333 1,-0.6666666667 1.5,-0.3333333333 1.5,0.3333333333 1,0.6666666667 0.5,0.3333333333 0,0.6666666667 -0.5,0.3333333333 -0.5,-0.3333333333\" fill=\"slategrey\" stroke=\"black\" stroke-width=\".05\"/></g>\n";
        o << "</defs>\n";
        for_rows(o, 0, m - 1, m, [&](Sink& row_out, int i) {
            for (int j = 1; j < 2 * m - 1; j += 2) {
                const double x = .5 * j + .5 * i;
                if ((t[(size_t)2 * i * n + j] & 4) == 4) use(row_out, "dR", x, i, true);
                if ((t[(size_t)2 * i * n + j] & 8) == 8) use(row_out, "dL", x, i, true);
                if ((t[(size_t)(2 * i + 1) * n + j] & 1) == 1) use(row_out, "dH", x, i, true);
            }
        });
        o << "</svg>";
        return finish(o);
    });
}

// TriangleDimerTiler::DimerToSVG(t, d) (:841-902); d = NULL takes the domain
// from the tiling (TilingToDomain).
rt_status rt_tridimer_dimer_svg(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!t || !filename) return RT_E_INVAL;
        const int n = side_of(tlen);
        Vec dom;
        if (!d) {
            int64_t len = 0;
            if (rt_tridimer_tiling_to_domain(t, tlen, nullptr, 0, &len) != RT_OK) return RT_E_INVAL;
            dom.resize((size_t)len);
            if (rt_tridimer_tiling_to_domain(t, tlen, dom.data(), len, &len) != RT_OK) return RT_E_INVAL;
            d = dom.data();
            dlen = len;
        }
        const int m = side_of(dlen / 2);
        // The domain of an n x n tiling is m x 2m with 2m = n; the loops below
        // read the tiling up to row and column 2m - 3.
        if (2 * (int64_t)m > n) return RT_E_INVAL;
        // The reference also reads one cell before the domain and one row past it.
        Vec pad((size_t)2 * m * (m + 2) + 2, 0);
        const int64_t cells = std::min<int64_t>(dlen, (int64_t)2 * m * m);
        for (int64_t k = 0; k < cells; ++k) pad[(size_t)k + 2 * m + 1] = d[k];
        auto D = [&](int i, int j) { return pad[(size_t)(i * 2 * m + j) + 2 * m + 1]; };
        Sink o(filename);
        tri_header(o, m);
        o << "<defs>\n";
        o << "<g id=\"dR\">  <polyline points= \".5,1 1,0\" stroke=\"darkblue\" stroke-width=\".05\"/> </g>\n";
        o << "<g id=\"dL\">  <polyline points= \".5,1 0,0\" stroke=\"darkred\" stroke-width=\".05\"/> </g>\n";
        o << "<g id=\"dH\">  <polyline points= \"1,0 0,0\" stroke=\"darkgreen\" stroke-width=\".05\"/> </g>\n";
        o << "<g id=\"eR\">  <polyline points= \".5,1 1,0\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"eL\">  <polyline points= \".5,1 0,0\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"eH\">  <polyline points= \"1,0 0,0\" stroke=\"black\" stroke-width=\".001\"/> </g>\n";
        o << "<g id=\"v1\">  <ellipse cx=\".5\" cy=\"0\" rx=\".1\" ry=\".1\" stroke=\"black\" stroke-width=\".02\" fill=\"black\"/> </g> \n";
        o << "<g id=\"v2\">  <ellipse cx=\"1.5\" cy=\"0\" rx=\".1\" ry=\".1\" stroke=\"black\" stroke-width=\".02\" fill=\"black\"/> </g> \n";
        o << "<g id=\"v3\">  <ellipse cx=\"1\" cy=\"1\" rx=\".1\" ry=\".1\" stroke=\"black\" stroke-width=\".02\" fill=\"black\"/> </g> \n";
        o << "</defs>\n";
        for_rows(o, 0, m - 1, 2 * m, [&](Sink& row_out, int i) {
            for (int j = 1; j < 2 * m - 1; j += 2) {
                const double x = .5 * j + .5 * i;
                const int32_t a = t[(size_t)2 * i * n + j], h = t[(size_t)(2 * i + 1) * n + j];
                if ((a & 4) == 4) use(row_out, "dR", x, i, true);
                else if (D(i, j - 1) == 1) use(row_out, "eR", x, i, true);
                if ((a & 8) == 8) use(row_out, "dL", x, i, true);
                else if (D(i, j - 1) == 1) use(row_out, "eL", x, i, true);
                if ((h & 1) == 1) use(row_out, "dH", x, i, true);
                else if (D(i, j - 1) == 1 || D(i - 1, j) == 1) use(row_out, "eH", x, i, true);
                if ((a & 4) == 0 && D(i, j) == 1) use(row_out, "eR", x, i, true);
                if ((a & 8) == 0 && D(i, j - 2) == 1 && j > 1) use(row_out, "eL", x, i, true);
            }
        });
        for_rows(o, 0, m, 2 * m, [&](Sink& row_out, int i) {
            for (int j = 2; j < 2 * m; j += 2) {
                const double x = .5 * j + .5 * i;
                if (D(i, j) == 1 || D(i, j - 1) == 1) use(row_out, "v1", x, i, true);
                if (D(i, j) == 1 || D(i, j + 1) == 1) use(row_out, "v2", x, i, true);
                if (D(i, j) == 1 || D(i, j + 1) == 1 || D(i, j - 1) == 1) use(row_out, "v3", x, i, true);
            }
        });
        o << "</svg>";
        return finish(o);
    });
}

// ---- text matrices (common.cpp:82-161) ---------------------------------------------------
// SaveMatrix: sqrt(size) rows of sqrt(size) values, each followed by a space.
rt_status rt_save_matrix(const int32_t* a, int64_t len, const char* filename) {
    return guarded([&]() -> rt_status {
        if (!a || !filename) return RT_E_INVAL;
        const int n = side_of(len);
        Sink o(filename);
        for_rows(o, 0, n, n, [&](Sink& row_out, int i) {
            for (int j = 0; j < n; ++j) row_out << a[(size_t)i * n + j] << " ";
            row_out << "\n";
        });
        return finish(o);
    });
}

// LoadMatrix: every maximal run of decimal digits is one value (like the
// reference, minus signs are not read).
rt_status rt_load_matrix(const char* filename, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!filename) return RT_E_INVAL;
        std::ifstream in(filename);
        if (!in) return RT_E_INVAL;
        std::vector<int32_t> v;
        char c;
        bool inside = false;
        // Digits accumulate modulo 2^64 (defined for any length); the value
        // kept is the low 32 bits, the wrap-around the reference's int
        // accumulator (common.cpp:149-155) shows in practice.
        uint64_t cur = 0;
        while (in.get(c)) {
            if (c >= '0' && c <= '9') {
                cur = inside ? cur * 10 + (uint64_t)(c - '0') : (uint64_t)(c - '0');
                inside = true;
            } else if (inside) {
                v.push_back((int32_t)(uint32_t)cur);
                inside = false;
            }
        }
        if (inside) v.push_back((int32_t)(uint32_t)cur);
        if (len) *len = (int64_t)v.size();
        if (!out) return RT_OK;
        if (cap < (int64_t)v.size()) return RT_E_INVAL;
        for (size_t k = 0; k < v.size(); ++k) out[k] = v[k];
        return RT_OK;
    });
}

// ---- binary matrices (no reference counterpart) ---------------------------------------------
// Header (little-endian, 40 bytes): "RTBMAT1\0", int64 count, int32 bits per
// value (1, 2, 4, 8, 16 or 32), int32 0, int64 base, uint64 FNV-1a of the
// payload.  Payload: value - base in `bits` bits, LSB first within each byte
// for bits < 8, little-endian words otherwise.  The smallest width that
// holds max - min is chosen, so a domino tiling (values 0..15) takes 4 bits
// a value, an eighth of the int32 array.
namespace {
const char kBinMagic[8] = {'R', 'T', 'B', 'M', 'A', 'T', '1', '\0'};
constexpr size_t kBinHeader = 40;

uint64_t fnv1a(const unsigned char* p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t k = 0; k < n; ++k) h = (h ^ p[k]) * 1099511628211ull;
    return h;
}

size_t bin_payload(int64_t count, int bits) { return (size_t)(((uint64_t)count * (uint64_t)bits + 7) / 8); }
}  // namespace

rt_status rt_save_matrix_binary(const int32_t* a, int64_t len, const char* filename) {
    return guarded([&]() -> rt_status {
        if ((!a && len > 0) || len < 0 || !filename) return RT_E_INVAL;
        int64_t lo = 0, hi = 0;
        for (int64_t k = 0; k < len; ++k) {
            if (k == 0 || a[k] < lo) lo = a[k];
            if (k == 0 || a[k] > hi) hi = a[k];
        }
        const uint64_t span = (uint64_t)(hi - lo);
        int bits = 32;
        for (int b : {1, 2, 4, 8, 16})
            if (span < (1ull << b)) {
                bits = b;
                break;
            }
        std::vector<unsigned char> pay(bin_payload(len, bits), 0);
        for (int64_t k = 0; k < len; ++k) {
            const uint32_t v = (uint32_t)((int64_t)a[k] - lo);
            if (bits < 8) {
                pay[(size_t)((k * bits) >> 3)] |= (unsigned char)(v << ((k * bits) & 7));
            } else {
                for (int byte = 0; byte < bits / 8; ++byte) pay[(size_t)k * (bits / 8) + byte] = (unsigned char)(v >> (8 * byte));
            }
        }
        unsigned char head[kBinHeader] = {0};
        std::memcpy(head, kBinMagic, 8);
        const uint64_t cnt = (uint64_t)len, base = (uint64_t)lo, sum = fnv1a(pay.data(), pay.size());
        for (int b = 0; b < 8; ++b) {
            head[8 + b] = (unsigned char)(cnt >> (8 * b));
            head[24 + b] = (unsigned char)(base >> (8 * b));
            head[32 + b] = (unsigned char)(sum >> (8 * b));
        }
        for (int b = 0; b < 4; ++b) head[16 + b] = (unsigned char)((uint32_t)bits >> (8 * b));
        std::FILE* f = std::fopen(filename, "wb");
        if (!f) return RT_E_INVAL;
        bool ok = std::fwrite(head, 1, kBinHeader, f) == kBinHeader &&
                  (pay.empty() || std::fwrite(pay.data(), 1, pay.size(), f) == pay.size());
        ok = (std::fclose(f) == 0) && ok;
        return ok ? RT_OK : RT_E_INVAL;
    });
}

rt_status rt_load_matrix_binary(const char* filename, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!filename) return RT_E_INVAL;
        std::FILE* f = std::fopen(filename, "rb");
        if (!f) return RT_E_INVAL;
        unsigned char head[kBinHeader];
        std::vector<unsigned char> pay;
        bool ok = std::fread(head, 1, kBinHeader, f) == kBinHeader && std::memcmp(head, kBinMagic, 8) == 0;
        uint64_t cnt = 0, base = 0, sum = 0;
        uint32_t bits = 0, zero = 0;
        if (ok) {
            for (int b = 0; b < 8; ++b) {
                cnt |= (uint64_t)head[8 + b] << (8 * b);
                base |= (uint64_t)head[24 + b] << (8 * b);
                sum |= (uint64_t)head[32 + b] << (8 * b);
            }
            for (int b = 0; b < 4; ++b) {
                bits |= (uint32_t)head[16 + b] << (8 * b);
                zero |= (uint32_t)head[20 + b] << (8 * b);
            }
            ok = zero == 0 && (bits == 1 || bits == 2 || bits == 4 || bits == 8 || bits == 16 || bits == 32) &&
                 cnt <= (1ull << 40);
        }
        if (ok) {
            // The file must hold exactly the payload its header announces; check
            // its size before the payload buffer is sized from the header.
            const size_t want = bin_payload((int64_t)cnt, (int)bits);
            const long at = std::ftell(f);
            ok = at == (long)kBinHeader && std::fseek(f, 0, SEEK_END) == 0 &&
                 std::ftell(f) == (long)(kBinHeader + want) && std::fseek(f, at, SEEK_SET) == 0;
            if (ok) {
                pay.resize(want);
                ok = pay.empty() || std::fread(pay.data(), 1, pay.size(), f) == pay.size();
                ok = ok && std::fgetc(f) == EOF && fnv1a(pay.data(), pay.size()) == sum;
            }
        }
        std::fclose(f);
        if (!ok) return RT_E_INVAL;  // not this format, truncated, trailing bytes or corrupted
        if (len) *len = (int64_t)cnt;
        if (!out) return RT_OK;
        if (cap < (int64_t)cnt) return RT_E_INVAL;
        const int64_t lo = (int64_t)base;
        for (uint64_t k = 0; k < cnt; ++k) {
            uint32_t v = 0;
            if (bits < 8) {
                v = (pay[(size_t)((k * bits) >> 3)] >> ((k * bits) & 7)) & ((1u << bits) - 1);
            } else {
                for (uint32_t byte = 0; byte < bits / 8; ++byte) v |= (uint32_t)pay[(size_t)k * (bits / 8) + byte] << (8 * byte);
            }
            out[k] = (int32_t)(lo + (int64_t)v);
        }
        return RT_OK;
    });
}

}  // extern "C"
