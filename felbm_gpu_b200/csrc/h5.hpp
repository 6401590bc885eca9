// Minimal HDF5 files without libhdf5 (no HDF5 library to link against):
// the file-format specification's version-0 superblock, one root group held
// as a symbol table (v1 B-tree + local heap + one symbol-table node), and
// datasets with version-1 object headers, contiguous layout, or (deflate >
// 0) one chunk per dataset through the deflate filter, as the reference
// writes its field files with output_deflate (felbm_gpu_main.cu:94-98:
// chunk = the whole dataset, gzip level = output_deflate). Enough for the
// reference's outputs (felbm_gpu_main.cu:86-189): fields, geometry,
// checkpoint and particle files of 1-D / 2-D arrays of little-endian
// double, float, int32 and uint32 values. The reader accepts files of this
// shape (the ones written here).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace fe {
namespace h5 {

enum Type { F64 = 0, F32 = 1, I32 = 2, U32 = 3 };

struct Dataset {
  std::string name;
  Type type = F64;
  std::vector<uint64_t> dims;   // 1 or 2 dimensions
  const void* data = nullptr;   // dims product elements of `type`
  int deflate = 0;              // 1-9: one chunk, deflate filter at this level
};

// Writes the datasets into a new file at path (at most 16); FE status.
int write(const std::string& path, const std::vector<Dataset>& sets);

struct Read {
  std::string name;
  Type type = F64;
  std::vector<uint64_t> dims;
  std::vector<unsigned char> bytes;
};

// Reads every dataset of a file written by write(); FE status.
int read(const std::string& path, std::vector<Read>& out);

}  // namespace h5
}  // namespace fe
