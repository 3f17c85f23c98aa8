// mplb_io.cu -- field files in the reference's per-rank formats.
//
// The reference's write step (multiPhasePP.c:289-301) calls
// writeScalarField / writeVectorField (src/IO/writeScalarField.c:10-59,
// src/IO/writeVectorField.c:9-70), which refuse a field holding a NaN and
// then dispatch on timeInfo.data (include/dataTypes.h:53):
//
//   asciiRaw   processor<pid>/<time>/<name>; scalar: "%g\n" per node
//              (asciiRaw/writeScalarToAsciiRaw.c:36); array: "%g " per
//              component and "\n" per node (asciiRaw/writeArrayToAsciiRaw.c:36-44)
//   binaryRaw  the same path; every value cast to float and written in node
//              order (binaryRaw/writeScalarToBinaryRaw.c:32-40,
//              binaryRaw/writeArrayToBinaryRaw.c:36-46)
//   pvtu       a DataArray block appended to processor<pid>/<time>/fields.vtu,
//              whose header (points, cells) the driver's writeMeshToVTK
//              writes before and whose footer writePvtuExtra writes after
//              (pvtu/writeScalarToPvtu.c:17-33, pvtu/writeArrayToPvtu.c:17-44)
//   ensight    MPI-IO, not provided here.
//
// The bytes are the reference's: the text is printed with the C library's
// "%g" (correctly rounded to six significant digits) and the binary form is
// the same float cast.  What differs is the work split: a field is cut into
// chunks of nodes that host threads format (or convert to float) in
// parallel, and the chunks are written in node order, so the file does not
// depend on the thread count.  Folders are made with mkdir(2), not a shell.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../../include/mplb_gpu.h"
#include "mplb_io.h"

int mplb_internal_fail(int code, const std::string& msg);

namespace {

int io_threads() {
    if (const char* e = std::getenv("MPLB_IO_THREADS")) {
        int v = std::atoi(e);
        if (v >= 1) return v < 256 ? v : 256;
    }
    unsigned c = std::thread::hardware_concurrency();
    return c == 0 ? 1 : (c < 32 ? (int)c : 32);
}

bool make_dirs(const std::string& path, std::string* err) {
    std::string cur;
    size_t i = 0;
    while (i <= path.size()) {
        size_t j = path.find('/', i);
        if (j == std::string::npos) j = path.size();
        cur = path.substr(0, j);
        if (!cur.empty() && cur != "." && cur != "..") {
            if (::mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) {
                *err = "Unable to create time folder " + cur + ": " + std::strerror(errno);
                return false;
            }
            struct stat st;
            if (::stat(cur.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) {
                *err = "Unable to create time folder " + cur;
                return false;
            }
        }
        i = j + 1;
    }
    return true;
}

enum class Text { Scalar, Array, PvtuScalar, PvtuArray };

// Nodes [a, b) of one field as text, appended to out.
void format_nodes(std::string& out, const double* v, uint64_t a, uint64_t b, uint32_t vs, Text t) {
    char buf[48];
    const bool pv = t == Text::PvtuScalar || t == Text::PvtuArray;
    const bool arr = t == Text::Array || t == Text::PvtuArray;
    for (uint64_t i = a; i < b; i++) {
        if (pv) out.append("          ", 10);
        const double* row = v + i * vs;
        for (uint32_t j = 0; j < vs; j++) {
            int k = std::snprintf(buf, sizeof buf, arr ? "%g " : "%g\n", row[j]);
            out.append(buf, (size_t)k);
        }
        if (arr) out.push_back('\n');
    }
}

// Writes nodes [0, n) in chunks formatted (or converted) by `threads`
// workers a round at a time; each round's chunks go to the file in order.
bool write_chunked(std::FILE* fp, const double* v, uint64_t n, uint32_t vs, bool binary, Text t, int threads,
                   std::string* err) {
    const uint64_t chunk = std::max<uint64_t>(1, (1u << 16) / vs);  // nodes per chunk
    const uint64_t nchunks = (n + chunk - 1) / chunk;
    if (threads > (int)nchunks) threads = (int)std::max<uint64_t>(nchunks, 1);
    const uint64_t per_round = (uint64_t)threads * 4;
    std::vector<std::string> text(binary ? 0 : per_round);
    std::vector<std::vector<float>> bin(binary ? per_round : 0);
    auto work = [&](uint64_t c0, uint64_t c1, int w) {
        for (uint64_t c = c0 + w; c < c1; c += threads) {
            const uint64_t a = c * chunk, b = std::min(n, a + chunk);
            const uint64_t slot = c - c0;
            if (binary) {
                std::vector<float>& o = bin[slot];
                o.resize((b - a) * vs);
                const double* s = v + a * vs;
                for (size_t k = 0; k < o.size(); k++) o[k] = (float)s[k];
            } else {
                std::string& o = text[slot];
                o.clear();
                format_nodes(o, v, a, b, vs, t);
            }
        }
    };
    for (uint64_t c0 = 0; c0 < nchunks; c0 += per_round) {
        const uint64_t c1 = std::min(nchunks, c0 + per_round);
        if (threads == 1) {
            work(c0, c1, 0);
        } else {
            // a worker that cannot be started leaves its chunks to this thread
            std::vector<std::thread> pool;
            std::vector<int> mine(1, 0);
            for (int w = 1; w < threads; w++) {
                try {
                    pool.emplace_back(work, c0, c1, w);
                } catch (...) {
                    mine.push_back(w);
                }
            }
            for (int w : mine) work(c0, c1, w);
            for (auto& th : pool) th.join();
        }
        for (uint64_t c = c0; c < c1; c++) {
            size_t want, got;
            if (binary) {
                const std::vector<float>& o = bin[c - c0];
                want = o.size();
                got = std::fwrite(o.data(), sizeof(float), want, fp);
            } else {
                const std::string& o = text[c - c0];
                want = o.size();
                got = std::fwrite(o.data(), 1, want, fp);
            }
            if (got != want) {
                *err = std::string("write failed: ") + std::strerror(errno);
                return false;
            }
        }
    }
    return true;
}

}  // namespace

int mplb_io_write(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                  const double* field, uint64_t n, uint32_t vsize, bool scalar, std::string* err) {
    if (!name || !*name || (!field && n)) {
        *err = "field name and values are required";
        return MPLB_E_ARG;
    }
    if (vsize == 0 || (scalar && vsize != 1)) {
        *err = "vsize must be 1 for a scalar field and at least 1 for an array";
        return MPLB_E_ARG;
    }
    if (std::strchr(name, '/')) {
        *err = "field name must not contain '/'";
        return MPLB_E_ARG;
    }
    if (format == MPLB_FMT_ENSIGHT) {
        *err = "EnSight output (MPI-IO) is not provided";
        return MPLB_E_UNSUPPORTED;
    }
    if (format != MPLB_FMT_ASCII_RAW && format != MPLB_FMT_BINARY_RAW && format != MPLB_FMT_PVTU) {
        *err = "unknown data format";
        return MPLB_E_ARG;
    }
    // writeScalarField.c:16-24 / writeVectorField.c:13-29: isnan only
    const uint64_t total = n * vsize;
    for (uint64_t i = 0; i < total; i++) {
        if (std::isnan(field[i])) {
            *err = std::string("Floating point exception. NaN solution (field ") + name + ")";
            return MPLB_E_NONFINITE;
        }
    }
    std::string dir = (root && *root) ? std::string(root) + "/" : std::string();
    dir += "processor" + std::to_string(pid) + "/" + std::to_string(time);
    std::string path;
    const char* mode;
    Text t;
    if (format == MPLB_FMT_PVTU) {
        path = dir + "/fields.vtu";
        mode = "a";
        t = scalar ? Text::PvtuScalar : Text::PvtuArray;
    } else {
        if (!make_dirs(dir, err)) return MPLB_E_IO;
        path = dir + "/" + name;
        mode = format == MPLB_FMT_BINARY_RAW ? "wb" : "w";
        t = scalar ? Text::Scalar : Text::Array;
    }
    std::FILE* fp = std::fopen(path.c_str(), mode);
    if (!fp) {
        *err = "cannot open " + path + ": " + std::strerror(errno);
        return MPLB_E_IO;
    }
    bool ok = true;
    if (format == MPLB_FMT_PVTU) {
        if (scalar)
            ok = std::fprintf(fp, "        <DataArray type=\"Float32\" Name=\"%s\" format=\"ascii\">\n", name) > 0;
        else
            ok = std::fprintf(fp, "        <DataArray type=\"Float32\" Name=\"%s\"  NumberOfComponents=\"%u\" format=\"ascii\">\n",
                              name, vsize) > 0;
        if (!ok) *err = "write failed: " + path;
    }
    if (ok) ok = write_chunked(fp, field, n, vsize, format == MPLB_FMT_BINARY_RAW, t, io_threads(), err);
    if (ok && format == MPLB_FMT_PVTU && std::fputs("        </DataArray>\n", fp) < 0) {
        ok = false;
        *err = "write failed: " + path;
    }
    if (std::fclose(fp) != 0 && ok) {
        ok = false;
        *err = "closing " + path + " failed: " + std::strerror(errno);
    }
    return ok ? 0 : MPLB_E_IO;
}

extern "C" int mplb_write_scalar_field(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                                       const double* field, uint64_t n) {
    std::string err;
    int rc = mplb_io_write(root, pid, time, format, name, field, n, 1, true, &err);
    return rc ? mplb_internal_fail(rc, err) : 0;
}

extern "C" int mplb_write_vector_field(const char* root, int32_t pid, uint32_t time, int32_t format, const char* name,
                                       const double* field, uint64_t n, uint32_t vsize) {
    std::string err;
    int rc = mplb_io_write(root, pid, time, format, name, field, n, vsize, false, &err);
    return rc ? mplb_internal_fail(rc, err) : 0;
}
