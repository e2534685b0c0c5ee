// .npy interchange (numax/io/npy.mojo): read what numpy.save wrote straight
// into device memory, and write device memory as numpy.save would.
//
// numax reads the whole file into a host List, then copies it to the device
// (npy.mojo:138-260, 349-453).  Here the payload streams: worker threads
// pread() fixed-size chunks into pinned staging buffers and each chunk goes
// to HBM by cudaMemcpyAsync while the next is being read, so a load runs at
// the file system's rate rather than a read followed by a copy.  A save runs
// the same pipeline the other way (device -> pinned -> pwrite()).
//
// The format is the documented one (numpy.lib.format, versions 1.0 and 2.0):
// the magic 0x93 'NUMPY', a version, a little-endian header length, an ASCII
// dict literal with the keys descr / fortran_order / shape, space padding to
// a 64-byte boundary and a newline, then the C-order payload.  What numax
// rejects is rejected with numax's wording (npy.mojo:179-250): bad magic (an
// .npz archive), versions other than 1.x / 2.x, a truncated header, a descr
// other than the requested one (big-endian named as such), Fortran order, a
// payload length that disagrees with the header, a rank or an extent other
// than the requested ones.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "nmx_common.cuh"
#include "nmx_la.h"

namespace nmx {
namespace npy {

// numpy's descr per NMX_* element code (the table of npy.mojo:76-114; one-byte
// types carry '|').  bfloat16 has no numpy dtype: empty.
struct Descr {
    const char *text;
    int itemsize;
};
constexpr Descr kDescr[] = {
    {"<f4", 4},  // NMX_F32
    {"<f8", 8},  // NMX_F64
    {"<f2", 2},  // NMX_F16
    {"|i1", 1},  // NMX_I8
    {"<i2", 2},  // NMX_I16
    {"<i4", 4},  // NMX_I32
    {"<i8", 8},  // NMX_I64
    {"|u1", 1},  // NMX_U8
    {"<u2", 2},  // NMX_U16
    {"<u4", 4},  // NMX_U32
    {"<u8", 8},  // NMX_U64
    {"|b1", 1},  // NMX_BOOL
    {"", 2},     // NMX_BF16
};
constexpr int kNumCodes = int(sizeof(kDescr) / sizeof(kDescr[0]));

// numpy's dtype names, for messages.
constexpr const char *kName[] = {"float32", "float64", "float16", "int8",   "int16",
                                 "int32",   "int64",   "uint8",   "uint16", "uint32",
                                 "uint64",  "bool",    "bfloat16"};

constexpr int kAlign = 64;           // numpy's ARRAY_ALIGN
constexpr int kGrowthDigits = 21;    // numpy's GROWTH_AXIS_MAX_DIGITS
constexpr size_t kChunk = 8u << 20;  // bytes per staged chunk
constexpr int kMaxThreads = 4;       // pread/pwrite workers per call

// Whether a file's descr names the same dtype as `want` (npy.mojo:455-481):
// '=' is native (little-endian) order; a one-byte type may carry '|', '<'
// or '='.
bool descr_matches(const std::string &file, const char *want) {
    if (file == want) return true;
    if (file.size() != 3 || std::strlen(want) != 3) return false;
    if (file[1] != want[1] || file[2] != want[2]) return false;
    const bool native = file[0] == '<' || file[0] == '=';
    if (file[2] == '1') return native || file[0] == '|';
    return native;
}

// The value of `key` in the header dict with spaces and quotes dropped: from
// the colon after the key to the next comma or newline at bracket depth zero
// (so the commas inside a shape tuple do not end it).  Empty when the key is
// absent (*found = false).
std::string dict_value(const std::string &h, const char *key, bool *found) {
    const std::string needle = std::string("'") + key + "'";
    size_t at = h.find(needle);
    *found = at != std::string::npos;
    if (!*found) return {};
    size_t colon = h.find(':', at + needle.size());
    if (colon == std::string::npos) {
        *found = false;
        return {};
    }
    std::string out;
    int depth = 0;
    for (size_t i = colon + 1; i < h.size(); ++i) {
        const char c = h[i];
        if (c == '(' || c == '[' || c == '{') {
            ++depth;
        } else if (c == ')' || c == ']' || c == '}') {
            if (depth == 0) break;
            --depth;
        } else if ((c == ',' || c == '\n') && depth == 0) {
            break;
        }
        if (c == ' ' || c == '\'' || c == '"') continue;
        out.push_back(c);
    }
    return out;
}

// Extents of a shape tuple's text, e.g. "(2,3)" -> {2, 3}, "()" -> {}.
bool parse_shape(const std::string &t, std::vector<int64_t> *dims) {
    dims->clear();
    int64_t v = 0;
    bool in = false;
    for (char c : t) {
        if (c >= '0' && c <= '9') {
            if (v > (INT64_MAX - 9) / 10) return false;
            v = v * 10 + (c - '0');
            in = true;
        } else if (in) {
            dims->push_back(v);
            v = 0;
            in = false;
        }
    }
    if (in) dims->push_back(v);
    return true;
}

struct Header {
    std::string descr;
    std::vector<int64_t> dims;
    int64_t offset = 0;         // payload start
    int64_t payload_bytes = 0;  // bytes the file holds after the header
    bool fortran = false;
};

// Read and validate the prelude and the dict of `fd` (everything but the
// descr / shape checks against the caller's request).  `who` prefixes the
// messages.  Returns 0 or NMX_ERR_IO / NMX_ERR_FORMAT.
int read_header(int fd, const char *who, Header *hd) {
    struct stat st;
    if (fstat(fd, &st) != 0) {
        set_error("%s: cannot stat the file: %s", who, std::strerror(errno));
        return NMX_ERR_IO;
    }
    const int64_t size = (int64_t)st.st_size;
    unsigned char pre[12];
    const ssize_t got = pread(fd, pre, sizeof(pre), 0);
    if (got < 10) {
        set_error("%s: file too short to be a .npy file", who);
        return NMX_ERR_FORMAT;
    }
    static const unsigned char magic[6] = {0x93, 'N', 'U', 'M', 'P', 'Y'};
    if (std::memcmp(pre, magic, 6) != 0) {
        set_error("%s: bad magic bytes -- not a .npy file. A .npz archive is a zip container, "
                  "not an .npy file: unzip it, or re-save each array with numpy.save",
                  who);
        return NMX_ERR_FORMAT;
    }
    const int major = pre[6];
    if (major != 1 && major != 2) {
        set_error("%s: unsupported .npy format version -- only the 1.x and 2.x headers are "
                  "understood",
                  who);
        return NMX_ERR_FORMAT;
    }
    int64_t hlen, hstart;
    if (major == 1) {
        hlen = (int64_t)pre[8] | ((int64_t)pre[9] << 8);
        hstart = 10;
    } else {
        if (got < 12) {
            set_error("%s: truncated .npy 2.x header", who);
            return NMX_ERR_FORMAT;
        }
        hlen = (int64_t)pre[8] | ((int64_t)pre[9] << 8) | ((int64_t)pre[10] << 16) |
               ((int64_t)pre[11] << 24);
        hstart = 12;
    }
    if (size < hstart + hlen) {
        set_error("%s: truncated .npy header", who);
        return NMX_ERR_FORMAT;
    }
    std::string h((size_t)hlen, '\0');
    if (hlen > 0 && pread(fd, &h[0], (size_t)hlen, hstart) != (ssize_t)hlen) {
        set_error("%s: cannot read the .npy header: %s", who, std::strerror(errno));
        return NMX_ERR_IO;
    }
    bool found = false;
    hd->descr = dict_value(h, "descr", &found);
    if (!found) {
        set_error("%s: .npy header has no 'descr' key", who);
        return NMX_ERR_FORMAT;
    }
    const std::string fo = dict_value(h, "fortran_order", &found);
    if (!found) {
        set_error("%s: .npy header has no 'fortran_order' key", who);
        return NMX_ERR_FORMAT;
    }
    hd->fortran = fo != "False";
    const std::string sh = dict_value(h, "shape", &found);
    if (!found) {
        set_error("%s: .npy header has no 'shape' key", who);
        return NMX_ERR_FORMAT;
    }
    if (!parse_shape(sh, &hd->dims)) {
        set_error("%s: malformed 'shape' entry", who);
        return NMX_ERR_FORMAT;
    }
    hd->offset = hstart + hlen;
    hd->payload_bytes = size - hd->offset;
    return 0;
}

// Elements of a shape, or -1 on int64 overflow.
int64_t element_count(const std::vector<int64_t> &dims) {
    int64_t n = 1;
    for (int64_t d : dims) {
        if (d != 0 && n > INT64_MAX / d) return -1;
        n *= d;
    }
    return n;
}

int code_of_descr(const std::string &d) {
    for (int c = 0; c < kNumCodes; ++c)
        if (kDescr[c].text[0] && descr_matches(d, kDescr[c].text)) return c;
    return -1;
}

// numpy.save's header bytes for (dtype, shape): the sorted-key dict, the
// growth padding numpy adds after it (21 - digits of the first extent, for
// rank >= 1), then spaces to a 64-byte boundary and a newline; version 1.0
// unless the length does not fit its 16-bit field, then 2.0.
std::string header_bytes(int code, int rank, const int64_t *shape) {
    std::string d = std::string("{'descr': '") + kDescr[code].text +
                    "', 'fortran_order': False, 'shape': (";
    for (int i = 0; i < rank; ++i) {
        d += std::to_string(shape[i]);
        if (i + 1 < rank) d += ", ";
    }
    if (rank == 1) d += ",";
    d += "), }";
    if (rank > 0) {
        const int digits = (int)std::to_string(shape[0]).size();
        if (digits < kGrowthDigits) d.append((size_t)(kGrowthDigits - digits), ' ');
    }
    std::string out;
    for (int version = 1; version <= 2; ++version) {
        const int prelude = version == 1 ? 10 : 12;
        const int64_t hlen = (int64_t)d.size() + 1;
        const int64_t pad = kAlign - ((prelude + hlen) % kAlign);
        const int64_t total = hlen + pad;
        if (version == 1 && total > 0xFFFF) continue;
        out.assign("\x93NUMPY", 6);
        out.push_back((char)version);
        out.push_back(0);
        for (int b = 0; b < (version == 1 ? 2 : 4); ++b) out.push_back((char)((total >> (8 * b)) & 0xFF));
        out += d;
        out.append((size_t)pad, ' ');
        out.push_back('\n');
        break;
    }
    return out;
}

// Pinned staging shared by a call's workers: two buffers per worker, each
// with the event of the copy that last used it.
struct Staging {
    std::vector<void *> buf;
    std::vector<cudaEvent_t> ev;
};

int staging_for(nmx_ctx ctx, int nbuf, Staging *s) {
    if ((int)ctx->npy_pinned.size() < nbuf) {
        while ((int)ctx->npy_pinned.size() < nbuf) {
            void *p = nullptr;
            cudaError_t e = cudaHostAlloc(&p, kChunk, cudaHostAllocDefault);
            if (e != cudaSuccess) {
                set_error("pinned staging cudaHostAlloc(%zu): %s", kChunk, cudaGetErrorString(e));
                return NMX_ERR_ALLOC;
            }
            cudaEvent_t ev = nullptr;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) {
                cudaFreeHost(p);
                set_error("staging event: %s", cudaGetErrorString(e));
                return NMX_ERR_CUDA;
            }
            ctx->npy_pinned.push_back(p);
            ctx->npy_event.push_back(ev);
        }
    }
    s->buf.assign(ctx->npy_pinned.begin(), ctx->npy_pinned.begin() + nbuf);
    s->ev.assign(ctx->npy_event.begin(), ctx->npy_event.begin() + nbuf);
    return 0;
}

int worker_count(int64_t bytes) {
    const int64_t chunks = (bytes + (int64_t)kChunk - 1) / (int64_t)kChunk;
    unsigned hw = std::thread::hardware_concurrency();
    int t = (int)std::min<int64_t>(chunks, std::min<int>(kMaxThreads, hw ? (int)hw : 1));
    return std::max(t, 1);
}

// Run body(worker, chunk) for chunks c = worker, worker + T, ... on T
// threads; the first nonzero status wins and stops the others at their next
// chunk.
template <typename F>
int run_chunks(int64_t bytes, int T, F body) {
    const int64_t chunks = (bytes + (int64_t)kChunk - 1) / (int64_t)kChunk;
    std::atomic<int> status{0};
    auto work = [&](int w) {
        int k = 0;
        for (int64_t c = w; c < chunks && status.load() == 0; c += T, ++k) {
            const int64_t off = c * (int64_t)kChunk;
            const size_t n = (size_t)std::min<int64_t>((int64_t)kChunk, bytes - off);
            const int rc = body(w, k & 1, off, n);
            if (rc != 0) {
                int zero = 0;
                status.compare_exchange_strong(zero, rc);
            }
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int w = 0; w < T; ++w) th.emplace_back(work, w);
        for (auto &t : th) t.join();
    }
    return status.load();
}

int full_pread(int fd, void *dst, size_t n, int64_t off) {
    char *p = static_cast<char *>(dst);
    while (n > 0) {
        const ssize_t r = pread(fd, p, n, off);
        if (r <= 0) return -1;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return 0;
}

int full_pwrite(int fd, const void *src, size_t n, int64_t off) {
    const char *p = static_cast<const char *>(src);
    while (n > 0) {
        const ssize_t r = pwrite(fd, p, n, off);
        if (r <= 0) return -1;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return 0;
}

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) close(fd);
    }
};

}  // namespace npy
}  // namespace nmx

using namespace nmx::npy;

extern "C" {

int nmx_npy_header(const char *path, int *dtype, int *rank, int64_t *shape, int max_rank,
                   int64_t *payload_offset) {
    NMX_ARG_CHECK(path != nullptr, 1, "path is NULL");
    NMX_ARG_CHECK(max_rank >= 0, 5, "max_rank < 0");
    NMX_ARG_CHECK(shape != nullptr || max_rank == 0, 4, "shape is NULL");
    const char *who = "numax.io.numpy.load";
    Fd f;
    f.fd = open(path, O_RDONLY | O_CLOEXEC);
    if (f.fd < 0) {
        nmx::set_error("%s: cannot open '%s': %s", who, path, std::strerror(errno));
        return NMX_ERR_IO;
    }
    Header hd;
    int rc = read_header(f.fd, who, &hd);
    if (rc) return rc;
    if (hd.descr.size() > 0 && hd.descr[0] == '>' && code_of_descr(hd.descr) < 0) {
        nmx::set_error("%s: big-endian .npy (descr '%s') -- nothing in numax byte-swaps; re-save "
                       "it native with arr.astype(arr.dtype.newbyteorder('<'))",
                       who, hd.descr.c_str());
        return NMX_ERR_FORMAT;
    }
    if (hd.fortran) {
        nmx::set_error("%s: Fortran-ordered .npy -- numax tensors are row-major; re-save with "
                       "numpy.ascontiguousarray(arr)",
                       who);
        return NMX_ERR_FORMAT;
    }
    const int code = code_of_descr(hd.descr);
    const int64_t count = element_count(hd.dims);
    if (code >= 0 && (count < 0 || count > INT64_MAX / kDescr[code].itemsize ||
                      hd.payload_bytes != count * kDescr[code].itemsize)) {
        nmx::set_error("%s: payload size doesn't match the header", who);
        return NMX_ERR_FORMAT;
    }
    if ((int)hd.dims.size() > max_rank) {
        nmx::set_error("%s: the file is rank %d, more than max_rank %d", who, (int)hd.dims.size(),
                       max_rank);
        return NMX_ERR_FORMAT;
    }
    if (dtype) *dtype = code;
    if (rank) *rank = (int)hd.dims.size();
    for (size_t i = 0; i < hd.dims.size(); ++i) shape[i] = hd.dims[i];
    if (payload_offset) *payload_offset = hd.offset;
    return 0;
}

int nmx_npy_load(nmx_ctx ctx, const char *path, int dtype, int rank, int64_t *shape, void *dst,
                 int64_t dst_bytes, void *stream) {
    NMX_ARG_CHECK(path != nullptr, 2, "path is NULL");
    NMX_ARG_CHECK(dtype >= 0 && dtype < kNumCodes, 3, "unknown dtype code");
    NMX_ARG_CHECK(rank >= 0 && rank <= NMX_NPY_MAX_RANK, 4, "rank out of range");
    NMX_ARG_CHECK(shape != nullptr || rank == 0, 5, "shape is NULL");
    NMX_ARG_CHECK(dst_bytes >= 0, 7, "dst_bytes < 0");
    const char *who = "numax.io.numpy.load";
    const Descr &want = kDescr[dtype];
    if (!want.text[0]) {
        nmx::set_error("%s: %s has no NumPy dtype, so no .npy file can hold it", who,
                       kName[dtype]);
        return NMX_ERR_FORMAT;
    }
    Fd f;
    f.fd = open(path, O_RDONLY | O_CLOEXEC);
    if (f.fd < 0) {
        nmx::set_error("%s: cannot open '%s': %s", who, path, std::strerror(errno));
        return NMX_ERR_IO;
    }
    Header hd;
    int rc = read_header(f.fd, who, &hd);
    if (rc) return rc;
    if (!descr_matches(hd.descr, want.text)) {
        if (!hd.descr.empty() && hd.descr[0] == '>')
            nmx::set_error("%s: big-endian .npy (descr '%s') -- nothing in numax byte-swaps; "
                           "re-save it native with arr.astype(arr.dtype.newbyteorder('<'))",
                           who, hd.descr.c_str());
        else
            nmx::set_error("%s: dtype mismatch -- the file holds '%s' but '%s' was requested", who,
                           hd.descr.c_str(), want.text);
        return NMX_ERR_FORMAT;
    }
    if (hd.fortran) {
        nmx::set_error("%s: Fortran-ordered .npy -- numax tensors are row-major; re-save with "
                       "numpy.ascontiguousarray(arr)",
                       who);
        return NMX_ERR_FORMAT;
    }
    const int64_t count = element_count(hd.dims);
    if (count < 0 || count > INT64_MAX / want.itemsize ||
        hd.payload_bytes != count * want.itemsize) {
        nmx::set_error("%s: payload size doesn't match the header", who);
        return NMX_ERR_FORMAT;
    }
    if ((int)hd.dims.size() != rank) {
        nmx::set_error("%s: rank mismatch -- the file is rank %d, rank %d was requested", who,
                       (int)hd.dims.size(), rank);
        return NMX_ERR_FORMAT;
    }
    for (int i = 0; i < rank; ++i) {
        if (shape[i] >= 0 && shape[i] != hd.dims[i]) {
            nmx::set_error("%s: shape mismatch", who);
            return NMX_ERR_FORMAT;
        }
    }
    const int64_t bytes = hd.payload_bytes;
    if (bytes > dst_bytes) {
        nmx::set_error("%s: the payload (%lld bytes) does not fit dst (%lld bytes)", who,
                       (long long)bytes, (long long)dst_bytes);
        return -7;
    }
    for (int i = 0; i < rank; ++i) shape[i] = hd.dims[i];
    if (bytes == 0) return 0;
    NMX_ARG_CHECK(dst != nullptr, 6, "dst is NULL");
    const int T = worker_count(bytes);
    const int fd = f.fd;
    char *out = static_cast<char *>(dst);
    if (ctx == nullptr) {
        // Host destination: the workers read straight into it.
        rc = run_chunks(bytes, T, [&](int, int, int64_t off, size_t n) {
            return full_pread(fd, out + off, n, hd.offset + off) == 0 ? 0 : NMX_ERR_IO;
        });
        if (rc) nmx::set_error("%s: read failed: %s", who, std::strerror(errno));
        return rc;
    }
    nmx::DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Staging s;
    NMX_TRY(staging_for(ctx, 2 * T, &s));
    rc = run_chunks(bytes, T, [&](int w, int k, int64_t off, size_t n) {
        const int b = 2 * w + k;
        // The copy that last read this buffer must have finished.
        if (cudaEventSynchronize(s.ev[b]) != cudaSuccess) return NMX_ERR_CUDA;
        if (full_pread(fd, s.buf[b], n, hd.offset + off) != 0) return NMX_ERR_IO;
        if (cudaMemcpyAsync(out + off, s.buf[b], n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaEventRecord(s.ev[b], st) != cudaSuccess)
            return NMX_ERR_CUDA;
        return 0;
    });
    const cudaError_t fin = cudaStreamSynchronize(st);
    if (rc == NMX_ERR_IO) {
        nmx::set_error("%s: read failed: %s", who, std::strerror(errno));
        return rc;
    }
    if (rc || fin != cudaSuccess) {
        nmx::set_error("%s: host-to-device copy failed: %s", who,
                       cudaGetErrorString(fin != cudaSuccess ? fin : cudaGetLastError()));
        return NMX_ERR_CUDA;
    }
    return 0;
}

int nmx_npy_save(nmx_ctx ctx, const char *path, int dtype, int rank, const int64_t *shape,
                 const void *src, void *stream) {
    NMX_ARG_CHECK(path != nullptr, 2, "path is NULL");
    NMX_ARG_CHECK(dtype >= 0 && dtype < kNumCodes, 3, "unknown dtype code");
    NMX_ARG_CHECK(rank >= 0 && rank <= NMX_NPY_MAX_RANK, 4, "rank out of range");
    NMX_ARG_CHECK(shape != nullptr || rank == 0, 5, "shape is NULL");
    const char *who = "numax.io.numpy.save";
    const Descr &d = kDescr[dtype];
    if (!d.text[0]) {
        nmx::set_error("%s: %s has no NumPy dtype, so it has no .npy representation", who,
                       kName[dtype]);
        return NMX_ERR_FORMAT;
    }
    std::vector<int64_t> dims(shape, shape + rank);
    for (int i = 0; i < rank; ++i) NMX_ARG_CHECK(shape[i] >= 0, 5, "negative extent");
    const int64_t count = element_count(dims);
    NMX_ARG_CHECK(count >= 0 && count <= INT64_MAX / d.itemsize, 5, "shape too large");
    const int64_t bytes = count * d.itemsize;
    NMX_ARG_CHECK(src != nullptr || bytes == 0, 6, "src is NULL");
    const std::string head = header_bytes(dtype, rank, shape);
    Fd f;
    f.fd = open(path, O_WRONLY | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
    if (f.fd < 0) {
        nmx::set_error("%s: cannot create '%s': %s", who, path, std::strerror(errno));
        return NMX_ERR_IO;
    }
    if (ftruncate(f.fd, (off_t)(head.size() + bytes)) != 0 ||
        full_pwrite(f.fd, head.data(), head.size(), 0) != 0) {
        nmx::set_error("%s: write failed: %s", who, std::strerror(errno));
        return NMX_ERR_IO;
    }
    if (bytes == 0) return 0;
    const int T = worker_count(bytes);
    const int fd = f.fd;
    const int64_t base = (int64_t)head.size();
    const char *in = static_cast<const char *>(src);
    int rc;
    if (ctx == nullptr) {
        rc = run_chunks(bytes, T, [&](int, int, int64_t off, size_t n) {
            return full_pwrite(fd, in + off, n, base + off) == 0 ? 0 : NMX_ERR_IO;
        });
        if (rc) nmx::set_error("%s: write failed: %s", who, std::strerror(errno));
        return rc;
    }
    nmx::DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Staging s;
    NMX_TRY(staging_for(ctx, 2 * T, &s));
    // Each worker keeps one copy ahead: chunk k's device-to-host copy is
    // queued before chunk k-1 is written out.
    const int64_t chunks = (bytes + (int64_t)kChunk - 1) / (int64_t)kChunk;
    std::atomic<int> status{0};
    std::atomic<int> io_fail{0};
    auto work = [&](int w) {
        auto span = [&](int64_t c, int64_t *off, size_t *n) {
            *off = c * (int64_t)kChunk;
            *n = (size_t)std::min<int64_t>((int64_t)kChunk, bytes - *off);
        };
        auto issue = [&](int64_t c, int b) {
            int64_t off;
            size_t n;
            span(c, &off, &n);
            if (cudaMemcpyAsync(s.buf[b], in + off, n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaEventRecord(s.ev[b], st) != cudaSuccess)
                return NMX_ERR_CUDA;
            return 0;
        };
        int k = 0;
        int64_t c = w;
        if (c < chunks) {
            const int r = issue(c, 2 * w);
            if (r) status = r;
        }
        for (; c < chunks && status.load() == 0; c += T, ++k) {
            const int b = 2 * w + (k & 1);
            if (c + T < chunks) {
                const int r = issue(c + T, 2 * w + ((k + 1) & 1));
                if (r) {
                    status = r;
                    break;
                }
            }
            if (cudaEventSynchronize(s.ev[b]) != cudaSuccess) {
                status = NMX_ERR_CUDA;
                break;
            }
            int64_t off;
            size_t n;
            span(c, &off, &n);
            if (full_pwrite(fd, s.buf[b], n, base + off) != 0) {
                io_fail = 1;
                status = NMX_ERR_IO;
                break;
            }
        }
    };
    // Staging buffers are shared with loads on this context: the caller's
    // device data must be complete, so the copies follow the work queued on
    // `stream`; every worker's copies are done before return.
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int w = 0; w < T; ++w) th.emplace_back(work, w);
        for (auto &t : th) t.join();
    }
    const cudaError_t fin = cudaStreamSynchronize(st);
    rc = status.load();
    if (io_fail.load()) {
        nmx::set_error("%s: write failed: %s", who, std::strerror(errno));
        return NMX_ERR_IO;
    }
    if (rc || fin != cudaSuccess) {
        nmx::set_error("%s: device-to-host copy failed: %s", who,
                       cudaGetErrorString(fin != cudaSuccess ? fin : cudaGetLastError()));
        return NMX_ERR_CUDA;
    }
    return 0;
}

}  // extern "C"
