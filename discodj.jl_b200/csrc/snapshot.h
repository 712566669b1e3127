// HDF5 snapshot writer shared by the host-array and the resident-state entry points.
#pragma once

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

namespace djb {

struct H5Array {
    std::string name;
    std::vector<uint64_t> dims;   // HDF5 (C-order) dimensions
    int elem;                     // 4 = float32, 8 = float64
};

struct H5Attr {
    std::string name;
    double value;                 // float64 scalar attribute of the root group
};

// Writes payload i (exactly the dataset's bytes) at the file position it is called at.
using H5Payload = std::function<int(size_t, FILE*)>;

// Writes a file with `arrays` as contiguous datasets of the root group and `attrs` as its
// attributes; the payloads are written in the order of `arrays`. Removes the file on error.
int h5_write_arrays(const char* path, const std::vector<H5Array>& arrays, const std::vector<H5Attr>& attrs,
                    const H5Payload& payload);

int h5_write_floats(FILE* fp, const float* p, size_t count);

}  // namespace djb
