// mriSolver input directory reader (0.2 binary and 1.0 text-header formats)
// and output writers.
//
// Formats, as read by the reference (kernels/structures.cpp):
//   0.2 (readDataFile, :782-863): float version, int dim1, int ncoils,
//       int nslices, int size, then float[size].
//   1.0 (readDataFile_10, :866-1162): "key = value" lines (version,
//       xDimension, yDimension, zDimension, coil_number, slice_number,
//       file_size), "//" comments, and any number of
//       "Binary_Size = n" + "Binary:" sections each followed by n float32;
//       "EOF" or the end of the file ends the header scan.
// Unlike the reference, malformed or truncated files are reported as
// IMP_ERR_FORMAT / IMP_ERR_IO instead of exiting the process.
#include "io.h"
#include "../../include/impatient_b200.h"

#include <cerrno>
#include <cmath>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>

namespace imp {

namespace {

struct File {
    FILE *f = nullptr;
    explicit File(const std::string &fn, const char *mode) { f = std::fopen(fn.c_str(), mode); }
    ~File() {
        if (f) std::fclose(f);
    }
};

bool read_line(FILE *f, std::string &line) {
    line.clear();
    int ch;
    bool any = false;
    while ((ch = std::fgetc(f)) != EOF) {
        any = true;
        if (ch == '\n') return true;
        line.push_back((char)ch);
    }
    return any;
}

std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r");
    return s.substr(a, b - a + 1);
}

int read_v02(FILE *f, const std::string &fn, DataFile &out, std::string &err) {
    float ver;
    int hdr[4];
    if (std::fread(&ver, 4, 1, f) != 1 || std::fread(hdr, 4, 4, f) != 4) {
        err = fn + ": truncated 0.2 header";
        return IMP_ERR_FORMAT;
    }
    out.version = ver;
    out.per_coil = hdr[0];
    out.coil_number = hdr[1];
    out.slice_number = hdr[2];
    const int size = hdr[3];
    if (size < 0 || hdr[0] < 0) {
        err = fn + ": negative size in 0.2 header";
        return IMP_ERR_FORMAT;
    }
    out.data.resize((size_t)size);
    if (size && std::fread(out.data.data(), 4, (size_t)size, f) != (size_t)size) {
        err = fn + ": data shorter than the stated size";
        return IMP_ERR_FORMAT;
    }
    return IMP_OK;
}

int read_v10(FILE *f, const std::string &fn, DataFile &out, std::string &err) {
    int file_size = -1;
    int local_coils = -1;
    size_t filled = 0;
    std::string line;
    while (read_line(f, line)) {
        std::string s = trim(line);
        if (s.empty() || s.compare(0, 2, "//") == 0) continue;
        if (s.compare(0, 3, "EOF") == 0) break;
        size_t eq = s.find('=');
        if (eq == std::string::npos) {
            err = fn + ": expected 'key = value', got '" + s + "'";
            return IMP_ERR_FORMAT;
        }
        std::string key = trim(s.substr(0, eq));
        std::string val = trim(s.substr(eq + 1));
        if (key == "version") {
            out.version = (float)std::atof(val.c_str());
        } else if (key == "xDimension") {
            out.nx = std::atoi(val.c_str());
        } else if (key == "yDimension") {
            out.ny = std::atoi(val.c_str());
        } else if (key == "zDimension") {
            out.nz = std::atoi(val.c_str());
        } else if (key == "coil_number") {
            local_coils = std::atoi(val.c_str());
            out.coil_number = local_coils;
        } else if (key == "slice_number") {
            out.slice_number = std::atoi(val.c_str());
        } else if (key == "file_size") {
            file_size = std::atoi(val.c_str());
            if (file_size < 0) {
                err = fn + ": negative file_size";
                return IMP_ERR_FORMAT;
            }
            if (local_coils <= 0) local_coils = 1;
            out.per_coil = file_size / local_coils;
            out.data.assign((size_t)file_size, 0.f);
        } else if (key == "Binary_Size") {
            if (file_size < 0) {
                err = fn + ": Binary_Size before file_size";
                return IMP_ERR_FORMAT;
            }
            const long n = std::atol(val.c_str());
            // the next non-empty, non-comment line must be "Binary:"
            bool found = false;
            while (read_line(f, line)) {
                std::string b = trim(line);
                if (b.empty() || b.compare(0, 2, "//") == 0) continue;
                if (b == "Binary:") found = true;
                break;
            }
            if (!found) {
                err = fn + ": Binary_Size not followed by Binary:";
                return IMP_ERR_FORMAT;
            }
            if (n < 0 || filled + (size_t)n > out.data.size()) {
                err = fn + ": binary sections exceed file_size";
                return IMP_ERR_FORMAT;
            }
            if (n && std::fread(out.data.data() + filled, 4, (size_t)n, f) != (size_t)n) {
                err = fn + ": binary section shorter than Binary_Size";
                return IMP_ERR_FORMAT;
            }
            filled += (size_t)n;
        }
        // unknown keys are ignored, as in the reference
    }
    if (file_size < 0) {
        err = fn + ": missing file_size";
        return IMP_ERR_FORMAT;
    }
    if (filled != (size_t)file_size) {
        err = fn + ": binary sections do not add up to file_size";
        return IMP_ERR_FORMAT;
    }
    return IMP_OK;
}

}  // namespace

int read_data_file(const std::string &fn, bool v02, DataFile &out, std::string &err) {
    File fp(fn, "rb");
    if (!fp.f) {
        err = fn + ": cannot open (" + std::strerror(errno) + ")";
        return IMP_ERR_IO;
    }
    out = DataFile();
    return v02 ? read_v02(fp.f, fn, out, err) : read_v10(fp.f, fn, out, err);
}

int read_mtx(const std::string &fn, SparseCoo &out, std::string &err) {
    out = SparseCoo();
    File fp(fn, "r");
    if (!fp.f) {
        err = fn + " not found";
        return IMP_ERR_IO;
    }
    char line[1024];
    if (!std::fgets(line, sizeof line, fp.f)) {
        err = fn + ": empty file";
        return IMP_ERR_FORMAT;
    }
    std::string banner(line);
    for (char &ch : banner) ch = (char)std::tolower((unsigned char)ch);
    if (banner.rfind("%%matrixmarket", 0) != 0) {
        err = fn + ": could not process Matrix Market banner";
        return IMP_ERR_FORMAT;
    }
    if (banner.find("coordinate") == std::string::npos || banner.find("matrix") == std::string::npos) {
        err = fn + ": only coordinate (sparse) matrices are supported";
        return IMP_ERR_FORMAT;
    }
    if (banner.find("complex") != std::string::npos) {
        err = fn + ": complex matrices are not supported";
        return IMP_ERR_FORMAT;
    }
    const bool pattern = banner.find("pattern") != std::string::npos;
    long rows = -1, cols = -1, nnz = -1;
    while (std::fgets(line, sizeof line, fp.f)) {
        if (line[0] == '%') continue;
        if (std::sscanf(line, "%ld %ld %ld", &rows, &cols, &nnz) == 3) break;
        bool blank = true;
        for (const char *c = line; *c; ++c)
            if (!std::isspace((unsigned char)*c)) blank = false;
        if (!blank) break;
    }
    if (rows <= 0 || cols <= 0 || nnz < 0 || rows > (1L << 30) || cols > (1L << 30) ||
        nnz > (1L << 30)) {
        err = fn + ": bad size line";
        return IMP_ERR_FORMAT;
    }
    out.rows = (int)rows;
    out.cols = (int)cols;
    out.row.resize(nnz);
    out.col.resize(nnz);
    out.val.resize(nnz);
    for (long e = 0; e < nnz; ++e) {
        long i = 0, j = 0;
        double v = 1.0;
        const int got = pattern ? std::fscanf(fp.f, "%ld %ld", &i, &j)
                                : std::fscanf(fp.f, "%ld %ld %lg", &i, &j, &v);
        if (got != (pattern ? 2 : 3)) {
            err = fn + ": failed to read entry " + std::to_string(e + 1);
            return IMP_ERR_FORMAT;
        }
        if (i < 1 || i > rows || j < 1 || j > cols) {
            err = fn + ": index out of range at entry " + std::to_string(e + 1);
            return IMP_ERR_FORMAT;
        }
        out.row[e] = (int)(i - 1);
        out.col[e] = (int)(j - 1);
        out.val[e] = (float)v;
    }
    return IMP_OK;
}

int load_input_dir(const std::string &dir, Dataset &ds, std::string &err) {
    ds = Dataset();
    float first = -1.f;
    {
        File fp(dir + "/kx.dat", "rb");
        if (!fp.f) {
            err = dir + "/kx.dat not found";
            return IMP_ERR_IO;
        }
        if (std::fread(&first, 4, 1, fp.f) != 1) {
            err = dir + "/kx.dat: empty file";
            return IMP_ERR_FORMAT;
        }
    }
    const bool v02 = first == 0.2f;
    struct Item {
        const char *name;
        std::vector<float> *dst;
        int *per_coil;
    };
    int kx_n = 0, ix_n = 0, sensi_n = 0, dummy = 0;
    // the reference's reading order (kernels/structures.cpp:650-700); the
    // coil and slice counts that stick are the last ones a file states
    Item items[] = {{"kx", &ds.kx, &kx_n},           {"ky", &ds.ky, &dummy},
                    {"kz", &ds.kz, &dummy},          {"kdata_r", &ds.kdata_r, &dummy},
                    {"kdata_i", &ds.kdata_i, &dummy}, {"sensi_r", &ds.sensi_r, &sensi_n},
                    {"sensi_i", &ds.sensi_i, &dummy}, {"fm", &ds.fm, &dummy},
                    {"ix", &ds.ix, &ix_n},           {"iy", &ds.iy, &dummy},
                    {"iz", &ds.iz, &dummy},          {"idata_r", &ds.idata_r, &dummy},
                    {"idata_i", &ds.idata_i, &dummy}, {"t", &ds.t, &dummy}};
    ds.num_coil = 1;
    ds.num_slices = 1;
    for (auto &it : items) {
        DataFile df;
        int st = read_data_file(dir + "/" + it.name + ".dat", v02, df, err);
        if (st != IMP_OK) return st;
        *it.per_coil = df.per_coil;
        if (df.coil_number >= 0) ds.num_coil = df.coil_number;
        if (df.slice_number >= 0) ds.num_slices = df.slice_number;
        if (df.nx >= 0) ds.nx = df.nx;
        if (df.ny >= 0) ds.ny = df.ny;
        if (df.nz >= 0) ds.nz = df.nz;
        ds.version = df.version;
        *it.dst = std::move(df.data);
    }
    ds.num_k = kx_n;
    ds.num_i = ix_n;
    if (ds.num_k <= 0 || ds.num_i <= 0 || ds.num_coil <= 0 || ds.num_slices <= 0) {
        err = dir + ": non-positive num_k / num_i / coils / slices";
        return IMP_ERR_FORMAT;
    }
    // One coil: sensitivities are forced to 1 (kernels/structures.cpp:710-716).
    if (ds.num_coil == 1) {
        for (int i = 0; i < sensi_n && i < (int)ds.sensi_r.size(); ++i) ds.sensi_r[i] = 1.f;
        for (int i = 0; i < sensi_n && i < (int)ds.sensi_i.size(); ++i) ds.sensi_i[i] = 0.f;
    }
    const size_t M = ds.num_k, N = ds.num_i, C = ds.num_coil, S = ds.num_slices;
    auto need = [&](const std::vector<float> &v, size_t n, const char *name) {
        if (v.size() < n) {
            err = dir + "/" + name + ".dat holds " + std::to_string(v.size()) +
                  " values, needs " + std::to_string(n);
            return false;
        }
        return true;
    };
    if (!need(ds.ky, M, "ky") || !need(ds.kz, M, "kz") || !need(ds.t, M, "t") ||
        !need(ds.iy, N, "iy") || !need(ds.iz, N, "iz") || !need(ds.kdata_r, S * C * M, "kdata_r") ||
        !need(ds.kdata_i, S * C * M, "kdata_i") || !need(ds.idata_r, S * N, "idata_r") ||
        !need(ds.idata_i, S * N, "idata_i") || !need(ds.fm, S * N, "fm") ||
        !need(ds.sensi_r, C * N, "sensi_r") || !need(ds.sensi_i, C * N, "sensi_i"))
        return IMP_ERR_FORMAT;
    return IMP_OK;
}

int export_text(const std::string &fn, const float *a, size_t n, std::string &err) {
    File fp(fn, "wt");
    if (!fp.f) {
        err = fn + ": cannot open for writing (" + std::strerror(errno) + ")";
        return IMP_ERR_IO;
    }
    for (size_t i = 0; i < n; ++i) std::fprintf(fp.f, "%f\n", a[i]);
    return IMP_OK;
}

int export_binary(const std::string &fn, const std::vector<const float *> &parts,
                  const std::vector<size_t> &sizes, std::string &err) {
    File fp(fn, "wb");
    if (!fp.f) {
        err = fn + ": cannot open for writing (" + std::strerror(errno) + ")";
        return IMP_ERR_IO;
    }
    for (size_t i = 0; i < parts.size(); ++i)
        if (sizes[i] && std::fwrite(parts[i], 4, sizes[i], fp.f) != sizes[i]) {
            err = fn + ": short write";
            return IMP_ERR_IO;
        }
    return IMP_OK;
}

int make_dirs(const std::string &dir, std::string &err) {
    if (dir.empty()) return IMP_OK;
    std::string cur;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!cur.empty()) {
                struct stat sb;
                if (stat(cur.c_str(), &sb) != 0 && mkdir(cur.c_str(), 0755) != 0 &&
                    errno != EEXIST) {
                    err = cur + ": cannot create directory (" + std::strerror(errno) + ")";
                    return IMP_ERR_IO;
                }
            }
        }
        if (i < dir.size()) cur.push_back(dir[i]);
    }
    return IMP_OK;
}

}  // namespace imp
