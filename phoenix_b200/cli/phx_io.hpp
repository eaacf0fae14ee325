// Matrix files of the PHOENIX command line: the text matrix, NumPy .npy, the
// PHOENIX binary (.ash) and MATLAB v4 (.mat) writers of
// FileHandler::outputMatrixToFile (source/system/filehandler.cpp:233-313) and
// PHOENIX::Output (include/misc/simple_binary.hpp), the text loaders
// (filehandler.cpp:160-231) and the column list loader (filehandler.cpp:392-417).
//
// The writers produce the reference's bytes for the same values, quirks
// included, so that tools reading its output read these files alike:
//   * text: "# SIZE <cols> <rows> LX .. LY .. DX .. DY .. TIME ..[ OSC T0 .. FREQ ..
//     SIGMA ..] :: PHOENIX_ MATRIX", the header numbers with six significant
//     digits, then every row as "v v ... \n" (each value followed by a space)
//     with fileout_precision significant digits (six when -1); a complex
//     matrix writes all real rows, then all imaginary rows;
//   * npy: magic 0x93 "NUMPY" 1 0, a dict header padded so that 10 + its
//     length + 1 is a multiple of 16, shape (rows, cols) of the requested
//     window (also when an increment thins it), little-endian data;
//   * ash: the npy layout with the magic name "PHOENIX" and the same padding
//     rule, always complex (a real matrix is written with zero imaginary parts);
//   * mat: a 128-byte text header, the five int32 fields with type 0 (double)
//     whatever the precision, the variable name "mat", column-major data
//     (real block, then imaginary block for complex matrices).
#pragma once

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

namespace phxio {

// FileHandler::Header (include/system/filehandler.hpp:31-70), in the build precision
template <typename T>
struct Header {
    T L_x = 0, L_y = 0, dx = 0, dy = 0, t = 0;
    T t0 = 0, freq = 0, sigma = 0;
};

// one number as an ostream with precision p and no floatfield prints it
inline std::string fmt_g(double v, int p) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.*g", p, v);
    return b;
}

template <typename T>
std::string header_text(const Header<T>& h) {
    std::string s = "LX " + fmt_g(h.L_x, 6) + " LY " + fmt_g(h.L_y, 6) + " DX " + fmt_g(h.dx, 6) + " DY " + fmt_g(h.dy, 6) +
                    " TIME " + fmt_g(h.t, 6);
    if (h.t0 != 0 && h.freq != 0 && h.sigma != 0)
        s += " OSC T0 " + fmt_g(h.t0, 6) + " FREQ " + fmt_g(h.freq, 6) + " SIGMA " + fmt_g(h.sigma, 6);
    return s;
}

// A window [c0, c1) x [r0, r1) of an N_c-wide row-major matrix, every inc-th
// point along both axes.
struct Window {
    uint32_t c0, c1, r0, r1, N_c, inc;
};

template <typename V, typename F>
void for_window(const Window& w, const V* buf, F f) {
    for (uint32_t i = w.r0; i < w.r1; i += w.inc)
        for (uint32_t j = w.c0; j < w.c1; j += w.inc) f(buf[j + (size_t)i * w.N_c]);
}

inline void put_bytes(std::string& out, const void* p, size_t n) { out.append(static_cast<const char*>(p), n); }

template <typename T>
const char* npy_descr(bool complex_) {
    if (std::is_same<T, float>::value) return complex_ ? "c8" : "f4";
    return complex_ ? "c16" : "f8";
}

// create_binary_header (simple_binary.hpp:55-86)
inline std::string binary_header(const std::string& descr, size_t rows, size_t cols, const std::string& magic_name) {
    std::string h = "{'descr': '<" + descr + "', 'fortran_order': False, 'shape': (" + std::to_string(rows) + ", " +
                    std::to_string(cols) + "), }";
    while ((10 + h.size()) % 16 != 15) h += ' ';
    h += '\n';
    std::string out;
    out += static_cast<char>(0x93);
    out += magic_name;
    out += static_cast<char>(0x01);
    out += static_cast<char>(0x00);
    const uint16_t len = static_cast<uint16_t>(h.size());
    out += static_cast<char>(len & 0xFF);
    out += static_cast<char>((len >> 8) & 0xFF);
    out += h;
    return out;
}

inline std::string mat_text_header(bool complex_) {
    std::string h(128, '\0');
    const char* text = complex_ ? "MATLAB 4.0 MAT-file, Created by PHOENIX::Output (complex)"
                                : "MATLAB 4.0 MAT-file, Created by PHOENIX::Output";
    std::memcpy(&h[0], text, std::strlen(text));
    return h;
}

inline void mat_array_header(std::string& out, uint32_t rows, uint32_t cols, int32_t imagf) {
    const int32_t f[5] = {0, (int32_t)rows, (int32_t)cols, imagf, 4};  // "mat" + NUL
    put_bytes(out, f, sizeof(f));
    put_bytes(out, "mat", 4);
}

// The bytes of one complex matrix file.  rows/cols of the headers are the
// window extents (r1 - r0, c1 - c0), as the reference writes them.
template <typename T>
std::string encode_complex(const std::string& type, const std::complex<T>* buf, const Window& w, const Header<T>& hd,
                           int precision) {
    const uint32_t rows = w.r1 - w.r0, cols = w.c1 - w.c0;
    std::vector<std::complex<T>> sub;
    for_window(w, buf, [&](const std::complex<T>& z) { sub.push_back(z); });
    std::string out;
    if (type == "npy" || type == "ash") {
        out = binary_header(npy_descr<T>(true), rows, cols, type == "npy" ? "NUMPY" : "PHOENIX");
        put_bytes(out, sub.data(), sub.size() * sizeof(std::complex<T>));
    } else if (type == "mat") {
        out = mat_text_header(true);
        mat_array_header(out, rows, cols, 1);
        // column-major real block, then imaginary block (rowMajorToColMajor of
        // a rows x cols buffer)
        for (int part = 0; part < 2; ++part)
            for (size_t j = 0; j < cols; ++j)
                for (size_t i = 0; i < rows; ++i) {
                    const size_t k = i * cols + j;
                    const T v = k < sub.size() ? (part ? sub[k].imag() : sub[k].real()) : T(0);
                    put_bytes(out, &v, sizeof(T));
                }
    } else {
        out = "# SIZE " + std::to_string(cols) + " " + std::to_string(rows) + " " + header_text(hd) + " :: PHOENIX_ MATRIX\n";
        const int p = precision != -1 ? precision : 6;
        for (int part = 0; part < 2; ++part)
            for (uint32_t i = w.r0; i < w.r1; i += w.inc) {
                for (uint32_t j = w.c0; j < w.c1; j += w.inc) {
                    const std::complex<T>& z = buf[j + (size_t)i * w.N_c];
                    out += fmt_g(part ? z.imag() : z.real(), p);
                    out += ' ';
                }
                out += '\n';
            }
    }
    return out;
}

template <typename T>
std::string encode_real(const std::string& type, const T* buf, const Window& w, const Header<T>& hd, int precision) {
    const uint32_t rows = w.r1 - w.r0, cols = w.c1 - w.c0;
    std::vector<T> sub;
    for_window(w, buf, [&](const T& v) { sub.push_back(v); });
    std::string out;
    if (type == "npy") {
        out = binary_header(npy_descr<T>(false), rows, cols, "NUMPY");
        put_bytes(out, sub.data(), sub.size() * sizeof(T));
    } else if (type == "ash") {
        out = binary_header(npy_descr<T>(true), rows, cols, "PHOENIX");
        for (const T& v : sub) {
            const std::complex<T> z(v, T(0));
            put_bytes(out, &z, sizeof(z));
        }
    } else if (type == "mat") {
        out = mat_text_header(false);
        mat_array_header(out, rows, cols, 0);
        for (size_t j = 0; j < cols; ++j)
            for (size_t i = 0; i < rows; ++i) {
                const size_t k = i * cols + j;
                const T v = k < sub.size() ? sub[k] : T(0);
                put_bytes(out, &v, sizeof(T));
            }
    } else {
        out = "# SIZE " + std::to_string(cols) + " " + std::to_string(rows) + " " + header_text(hd) + " :: PHOENIX_ MATRIX\n";
        const int p = precision != -1 ? precision : 6;
        for (uint32_t i = w.r0; i < w.r1; i += w.inc) {
            for (uint32_t j = w.c0; j < w.c1; j += w.inc) {
                out += fmt_g(buf[j + (size_t)i * w.N_c], p);
                out += ' ';
            }
            out += '\n';
        }
    }
    return out;
}

inline bool write_file(const std::string& path, const std::string& bytes) {
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) return false;
    f.write(bytes.data(), (std::streamsize)bytes.size());
    return (bool)f;
}

// FileHandler::loadMatrixFromFile for complex buffers: the header's third and
// fourth tokens are N_c and N_r; then the real block, then the imaginary
// block, lines starting with '#' and empty lines skipped.  Returns the number
// of values read, -1 when the file cannot be opened.
template <typename T>
long long load_complex_txt(const std::string& path, std::vector<std::complex<T>>& out, uint32_t& N_c, uint32_t& N_r) {
    std::ifstream f(path);
    if (!f.is_open()) return -1;
    std::string line, tok;
    std::getline(f, line);
    {
        std::istringstream is(line);
        N_c = N_r = 0;
        is >> tok >> tok >> N_c >> N_r;
    }
    const size_t N = (size_t)N_c * N_r;
    out.assign(N, std::complex<T>(0, 0));
    size_t i = 0;
    T v;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream is(line);
        if (i < N) {
            while (is >> v) {
                if (i < N) out[i] = std::complex<T>(v, 0);
                ++i;
            }
        } else {
            while (is >> v) {
                if (i - N < N) out[i - N] = std::complex<T>(out[i - N].real(), v);
                ++i;
            }
        }
    }
    return (long long)i;
}

// FileHandler::loadListFromFile: whitespace-separated columns, '#' lines skipped
template <typename T>
std::vector<std::vector<T>> load_list(const std::string& path) {
    std::vector<std::vector<T>> data;
    std::ifstream f(path);
    if (!f.is_open()) return data;
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream is(line);
        T v;
        size_t col = 0;
        while (is >> v) {
            if (data.size() <= col) data.emplace_back();
            data[col].push_back(v);
            ++col;
        }
    }
    return data;
}

}  // namespace phxio
