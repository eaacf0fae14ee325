// C entry points of the command line's file formats and envelope evaluation
// (libphx_io.so), for tests and for callers that write PHOENIX matrices.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "phx_envelope.hpp"
#include "phx_io.hpp"

using namespace phxio;

namespace {

template <typename T>
long long encode(const char* type, int is_complex, const void* data, uint32_t N_c, uint32_t N_r, const uint32_t* win,
                 const double* h8, int precision, char** out) {
    Header<T> hd{(T)h8[0], (T)h8[1], (T)h8[2], (T)h8[3], (T)h8[4], (T)h8[5], (T)h8[6], (T)h8[7]};
    const Window w{win[0], win[1], win[2], win[3], N_c, win[4]};
    (void)N_r;
    const std::string b = is_complex ? encode_complex<T>(type, static_cast<const std::complex<T>*>(data), w, hd, precision)
                                     : encode_real<T>(type, static_cast<const T*>(data), w, hd, precision);
    *out = static_cast<char*>(std::malloc(b.size() ? b.size() : 1));
    if (!*out) return -1;
    std::memcpy(*out, b.data(), b.size());
    return (long long)b.size();
}

template <typename T>
int envelope(int argc, const char** argv, const char* family, int group, int pol, double dflt, void* out, char* err, int errlen) {
    try {
        Args a;
        a.v.assign(argv, argv + argc);
        uint32_t N_c = 400, N_r = 400;
        T L_x = 100, L_y = 100;
        int i;
        if ((i = a.find({"N", "gridsize"}, 0, "--")) != -1) {
            N_c = (uint32_t)(int)a.num(++i, "N_c");
            N_r = (uint32_t)(int)a.num(i, "N_r");
        }
        if ((i = a.find({"L", "gridlength", "xmax"}, 0, "--")) != -1) {
            L_x = (T)a.num(++i, "L");
            L_y = (T)a.num(i, "L");
        }
        const std::string f = family;
        std::vector<std::string> keys{f};
        if (f == "initState") keys = {"initState", "initialState", "iS"};
        if (f == "initReservoir") keys = {"initReservoir", "initialReservoir", "iR"};
        const bool time = f == "pump" || f == "potential" || f == "pulse";
        Envelope<T> e = Envelope<T>::parse(a, keys, time);
        typename Envelope<T>::Dims d{N_c, N_r, L_x, L_y, L_x / (T)(N_c - 1), L_y / (T)(N_r - 1)};
        std::vector<std::complex<T>> b((size_t)N_c * N_r);
        std::string msg;
        if (!e.calculate(b.data(), group, (uint32_t)pol, d, (T)dflt, msg)) throw std::runtime_error(msg);
        std::memcpy(out, b.data(), b.size() * sizeof(std::complex<T>));
        return e.group_size();
    } catch (const std::exception& ex) {
        if (err && errlen > 0) {
            std::strncpy(err, ex.what(), (size_t)errlen - 1);
            err[errlen - 1] = 0;
        }
        return -1;
    }
}

}  // namespace

extern "C" {

// The bytes of one matrix file ("txt", "npy", "ash", "mat") as the command
// line writes it.  dtype 0 = float, 1 = double; win = {c0, c1, r0, r1, inc};
// header8 = {L_x, L_y, dx, dy, t, t0, freq, sigma}.  Returns the length and a
// malloc'ed buffer in *out (free with phxio_free), -1 on failure.
__attribute__((visibility("default"))) long long phxio_encode(const char* type, int dtype, int is_complex, const void* data,
                                                              uint32_t N_c, uint32_t N_r, const uint32_t* win,
                                                              const double* header8, int precision, char** out) {
    if (!type || !data || !win || !header8 || !out) return -1;
    return dtype == 0 ? encode<float>(type, is_complex, data, N_c, N_r, win, header8, precision, out)
                      : encode<double>(type, is_complex, data, N_c, N_r, win, header8, precision, out);
}

__attribute__((visibility("default"))) void phxio_free(void* p) { std::free(p); }

// One envelope family of a command line (--pump, --potential, --pulse,
// --fftMask, --initState, --initReservoir) evaluated on the grid of its
// --N / --L: complex N_r x N_c values into out (dtype 0 = float pairs,
// 1 = double pairs); group < 0 = all groups; pol 1 = plus, 2 = minus,
// 3 = both.  Returns the number of temporal groups, -1 on error (message in err).
__attribute__((visibility("default"))) int phxio_envelope(int argc, const char** argv, const char* family, int dtype,
                                                          int group, int pol, double dflt, void* out, char* err,
                                                          int errlen) {
    if (!argv || !family || !out) return -1;
    return dtype == 0 ? envelope<float>(argc, argv, family, group, pol, dflt, out, err, errlen)
                      : envelope<double>(argc, argv, family, group, pol, dflt, out, err, errlen);
}

}  // extern "C"
