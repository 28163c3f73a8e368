// Readers and writers for the mriSolver input directory and output files.
#pragma once
#include <string>
#include <vector>

namespace imp {

// One input file.  Fields that the file does not state keep -1.
struct DataFile {
    float version = -1.f;
    int per_coil = 0;        // elements per coil ("dims[0]" of the reference)
    int coil_number = -1;    // stated coil count (0.2: always stated)
    int slice_number = -1;
    int nx = -1, ny = -1, nz = -1;
    std::vector<float> data;
};

// The reference's loadInputData() result (kernels/structures.cpp:569-780).
struct Dataset {
    float version = 0.f;
    int num_k = 0, num_i = 0, num_coil = 1, num_slices = 1;
    int nx = 0, ny = 0, nz = 0;  // 1.0 headers only
    std::vector<float> kx, ky, kz, ix, iy, iz, t, fm;
    std::vector<float> kdata_r, kdata_i, idata_r, idata_i, sensi_r, sensi_i;
};

// Both return an imp_status code; `err` receives a message on failure.
int read_data_file(const std::string &fn, bool v02, DataFile &out, std::string &err);
int load_input_dir(const std::string &dir, Dataset &ds, std::string &err);

// A sparse matrix read from a Matrix Market coordinate file (c.rmtx), 0-based.
struct SparseCoo {
    int rows = 0, cols = 0;
    std::vector<int> row, col;
    std::vector<float> val;
};

// readMtxFile() of kernels/mmio.cpp:668-830: banner "%%MatrixMarket matrix
// coordinate real|integer|pattern general", '%' comment lines, "rows cols nnz",
// then nnz lines "i j value" (1-based; pattern files have no value: 1.0).
// Complex matrices are refused, as by the reference.
int read_mtx(const std::string &fn, SparseCoo &out, std::string &err);

// "%f\n" per element (kernels/structures.cpp:1165-1175).
int export_text(const std::string &fn, const float *a, size_t n, std::string &err);
// Raw float32 array (the Toeplitz out.file / FhD.file layout).
int export_binary(const std::string &fn, const std::vector<const float *> &parts,
                  const std::vector<size_t> &sizes, std::string &err);

int make_dirs(const std::string &dir, std::string &err);

}  // namespace imp
