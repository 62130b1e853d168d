// hj_ingest.cpp -- dataset ingest: the reference's text format parsed in
// parallel, and a binary twin that reads back the identical values.
//
// Reference counterpart: importNDDataset (import_dataset.cpp:10-40).  It reads
// the whole file as tokens split at every ',' (getline with ',' as the
// delimiter, so newlines are not separators on their own), and from each
// token extracts values with `stringstream >> DTYPE` until an extraction
// fails, dropping the rest of that token; main.cu keeps the first
// floor(values / GPUNUMDIM) * GPUNUMDIM values as points.  One extraction is
// libstdc++'s num_get for floating point in the C locale:
//   * leading whitespace skipped (the stream's skipws);
//   * the longest prefix of  [+-]? digits* ('.' digits*)? ([eE] [+-]? digits*)?
//     accumulated, where the exponent is taken only after a mantissa digit
//     and no '.' after it;
//   * that text converted with strtof / strtod ("C" locale); the extraction
//     fails when the conversion does not use all of it, or overflows to inf.
// hj_import_text applies exactly these rules, with the file cut into chunks at
// comma boundaries (a token never spans two chunks) parsed by OpenMP threads
// and concatenated in file order, so it yields the same values in the same
// order: bit for bit, since both end in glibc's correctly rounded strtof/strtod.
//
// The binary twin: a 32-byte header ("HJDS0001", dataset type, d, n) then the
// n x d values, little-endian.  hj_import_binary also reads the reference's
// raw binary layout (importNDDatasetBinary, import_dataset.cpp:63-100: the
// values only, n from the file size).
#include <algorithm>
#include <clocale>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <locale.h>
#include <omp.h>
#include <string>
#include <vector>

#include "hegjoin_b200.h"

namespace hj {
void set_error(const char* fmt, ...);
}

namespace {

locale_t c_locale() {
    static locale_t loc = newlocale(LC_ALL_MASK, "C", (locale_t)0);
    return loc;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

inline bool convert(const char* s, float* v) {
    char* e = nullptr;
    const float x = strtof_l(s, &e, c_locale());
    if (e == s || *e != '\0' || std::isinf(x)) return false;
    *v = x;
    return true;
}
inline bool convert(const char* s, double* v) {
    char* e = nullptr;
    const double x = strtod_l(s, &e, c_locale());
    if (e == s || *e != '\0' || std::isinf(x)) return false;
    *v = x;
    return true;
}

// One `>>` extraction from [p, end): the value and the position after the
// characters it consumed, or nullptr when it fails.
template <typename T>
const char* extract(const char* p, const char* end, T* out, std::string& buf) {
    buf.clear();
    const char* q = p;
    if (q < end && (*q == '+' || *q == '-')) buf += *q++;
    bool mantissa = false, dec = false, sci = false;
    while (q < end) {
        const char c = *q;
        if (!dec && !sci && c == '.') {
            buf += '.';
            dec = true;
        } else if (c >= '0' && c <= '9') {
            buf += c;
            mantissa = true;
        } else if ((c == 'e' || c == 'E') && !sci && mantissa) {
            buf += 'e';
            sci = true;
            ++q;
            if (q < end && (*q == '+' || *q == '-')) buf += *q++;
            continue;
        } else {
            break;
        }
        ++q;
    }
    if (buf.empty() || !convert(buf.c_str(), out)) return nullptr;
    return q;
}

// Values of the tokens in [p, end), which starts at a token boundary and ends
// at one (just after a ',' or at the file's end).
template <typename T>
void parse_range(const char* p, const char* end, std::vector<T>& vals) {
    std::string buf;
    while (p < end) {
        const char* tok_end = static_cast<const char*>(std::memchr(p, ',', (size_t)(end - p)));
        if (!tok_end) tok_end = end;
        for (;;) {
            while (p < tok_end && is_space(*p)) ++p;
            if (p == tok_end) break;
            T v;
            const char* q = extract<T>(p, tok_end, &v, buf);
            if (!q) break;   // the rest of the token is dropped, as the stream's failbit ends the loop
            vals.push_back(v);
            p = q;
        }
        p = tok_end + (tok_end < end ? 1 : 0);
    }
}

hj_status read_file(const char* path, std::vector<char>& data) {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        hj::set_error("cannot open %s", path);
        return HJ_ERR_INVALID;
    }
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0) {
        std::fclose(f);
        hj::set_error("cannot size %s", path);
        return HJ_ERR_INVALID;
    }
    data.resize((size_t)size);
    const size_t got = size ? std::fread(data.data(), 1, (size_t)size, f) : 0;
    std::fclose(f);
    if (got != (size_t)size) {
        hj::set_error("short read of %s", path);
        return HJ_ERR_INVALID;
    }
    return HJ_OK;
}

template <typename T>
hj_status import_text_t(const char* path, uint32_t d, void** out, uint64_t* n_points) {
    std::vector<char> data;
    hj_status s = read_file(path, data);
    if (s != HJ_OK) return s;
    const char* base = data.data();
    const size_t size = data.size();
    // chunks start just after a comma (or at 0) and end at the next chunk's start
    const int nt = omp_get_max_threads();
    const size_t nchunks = size < (1u << 20) ? 1 : (size_t)nt * 4;
    std::vector<size_t> cut(nchunks + 1, size);
    cut[0] = 0;
    for (size_t i = 1; i < nchunks; ++i) {
        size_t pos = std::max(cut[i - 1], size / nchunks * i);
        const void* c = pos < size ? std::memchr(base + pos, ',', size - pos) : nullptr;
        cut[i] = c ? (size_t)(static_cast<const char*>(c) - base) + 1 : size;
    }
    std::vector<std::vector<T>> parts(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < (long long)nchunks; ++i) {
        parts[i].reserve((cut[i + 1] - cut[i]) / 8 + 16);
        parse_range<T>(base + cut[i], base + cut[i + 1], parts[i]);
    }
    std::vector<size_t> off(nchunks + 1, 0);
    for (size_t i = 0; i < nchunks; ++i) off[i + 1] = off[i] + parts[i].size();
    const uint64_t np = off[nchunks] / d;   // trailing values that do not fill a point are dropped (main.cu)
    T* vals = static_cast<T*>(std::malloc(std::max<size_t>(1, (size_t)np * d) * sizeof(T)));
    if (!vals) {
        hj::set_error("host allocation of %llu values failed", (unsigned long long)(np * d));
        return HJ_ERR_OOM;
    }
    const size_t keep = (size_t)np * d;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < (long long)nchunks; ++i) {
        if (off[i] >= keep) continue;
        const size_t m = std::min(parts[i].size(), keep - off[i]);
        std::memcpy(vals + off[i], parts[i].data(), m * sizeof(T));
    }
    *out = vals;
    *n_points = np;
    return HJ_OK;
}

constexpr char kMagic[8] = {'H', 'J', 'D', 'S', '0', '0', '0', '1'};

struct BinHeader {
    char magic[8];
    uint32_t dtype;
    uint32_t d;
    uint64_t n;
    uint64_t reserved;
};
static_assert(sizeof(BinHeader) == 32, "binary header is 32 bytes");

}  // namespace

extern "C" {

hj_status hj_import_text(const char* path, uint32_t d, int dtype, void** h_values, uint64_t* n_points) {
    if (!path || !h_values || !n_points || d == 0 || (dtype != HJ_F32 && dtype != HJ_F64)) {
        hj::set_error("hj_import_text: invalid arguments");
        return HJ_ERR_INVALID;
    }
    *h_values = nullptr;
    *n_points = 0;
    return dtype == HJ_F32 ? import_text_t<float>(path, d, h_values, n_points)
                           : import_text_t<double>(path, d, h_values, n_points);
}

hj_status hj_write_binary(const char* path, const void* h_values, uint64_t n_points, uint32_t d, int dtype) {
    if (!path || (!h_values && n_points) || d == 0 || (dtype != HJ_F32 && dtype != HJ_F64)) {
        hj::set_error("hj_write_binary: invalid arguments");
        return HJ_ERR_INVALID;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        hj::set_error("cannot create %s", path);
        return HJ_ERR_INVALID;
    }
    BinHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.dtype = (uint32_t)dtype;
    h.d = d;
    h.n = n_points;
    const size_t bytes = (size_t)n_points * d * (dtype == HJ_F64 ? 8 : 4);
    const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && (bytes == 0 || std::fwrite(h_values, 1, bytes, f) == bytes);
    if (std::fclose(f) != 0 || !ok) {
        hj::set_error("write to %s failed", path);
        return HJ_ERR_INVALID;
    }
    return HJ_OK;
}

hj_status hj_import_binary(const char* path, uint32_t d, int dtype, void** h_values, uint64_t* n_points) {
    if (!path || !h_values || !n_points || d == 0 || (dtype != HJ_F32 && dtype != HJ_F64)) {
        hj::set_error("hj_import_binary: invalid arguments");
        return HJ_ERR_INVALID;
    }
    *h_values = nullptr;
    *n_points = 0;
    std::vector<char> data;
    hj_status s = read_file(path, data);
    if (s != HJ_OK) return s;
    const size_t es = dtype == HJ_F64 ? 8 : 4;
    size_t first = 0;
    uint64_t n = 0;
    if (data.size() >= sizeof(BinHeader) && std::memcmp(data.data(), kMagic, 8) == 0) {
        BinHeader h;
        std::memcpy(&h, data.data(), sizeof(h));
        if (h.dtype != (uint32_t)dtype || h.d != d) {
            hj::set_error("hj_import_binary: %s holds dtype %u, d = %u (asked for %d, %u)", path, h.dtype, h.d, dtype, d);
            return HJ_ERR_INVALID;
        }
        if (data.size() - sizeof(BinHeader) < (size_t)h.n * d * es) {
            hj::set_error("hj_import_binary: %s is truncated", path);
            return HJ_ERR_INVALID;
        }
        first = sizeof(BinHeader);
        n = h.n;
    } else {
        n = data.size() / es / d;   // the reference's raw layout: values only
    }
    void* vals = std::malloc(std::max<size_t>(1, (size_t)n * d * es));
    if (!vals) {
        hj::set_error("host allocation failed");
        return HJ_ERR_OOM;
    }
    std::memcpy(vals, data.data() + first, (size_t)n * d * es);
    *h_values = vals;
    *n_points = n;
    return HJ_OK;
}

void hj_host_free(void* p) { std::free(p); }

}  // extern "C"
