// h5mini.h -- a small HDF5 reader/writer for the x1 command line and the
// accuracy post-processor (no libhdf5 on the target hosts).
//
// Written from the HDF5 file format specification (version 3.0 of the
// spec document; the formats themselves date from HDF5 1.8/1.10):
//
// * reads  superblock versions 0-3; object headers v1 and v2 with
//          continuation blocks; groups with a symbol table (v1 B-tree +
//          local heap) or compact link messages; datasets of 8/16/32/64-bit
//          integers or 32/64-bit IEEE floats, little endian, contiguous or
//          compact layout (layout messages v1-v4), no filters;
// * writes the classic format libhdf5 produces with its default (earliest)
//          library-version bounds: superblock v0, object headers v1,
//          symbol-table groups; new files, or groups and datasets added to
//          an existing file of that format (appended at the end of the
//          file; the parent's symbol table is rebuilt and relinked).
//
// Datasets are what H5LTmake_dataset_{int,double} makes: a simple dataspace
// of the given dims (C order), NATIVE_INT (32-bit LE) or NATIVE_DOUBLE.
#ifndef GJX_H5MINI_H
#define GJX_H5MINI_H

#include <cstdint>
#include <string>
#include <vector>

namespace h5m {

struct Array {
  std::vector<uint64_t> dims; // C order
  int cls = 0;                // 0 integer, 1 float
  unsigned size = 0u;         // bytes per element
  bool is_signed = true;
  std::vector<uint8_t> raw;   // dims product * size bytes, little endian
  uint64_t count() const;
  bool to_double(std::vector<double> &out) const;
  bool to_int(std::vector<int> &out) const;
};

// read the dataset at path "group/name" (any depth); false and err on failure
bool read(const std::string &file, const std::string &path, Array &out, std::string &err);
// whether the object at path exists (group or dataset)
bool exists(const std::string &file, const std::string &path, std::string &err);

struct NewDataset {
  std::string name;
  std::vector<uint64_t> dims;
  bool is_float = true; // double, else 32-bit signed int
  const void *data = nullptr;
};

// Write the datasets into group `group` (one level below the root) of `file`.
//   mode 0: create a new file (fails if it exists), then the group;
//   mode 1: the file exists: create the group (fails if it exists);
//   mode 2: the file exists: create the group if absent; a dataset that
//           exists already with the same type and dims is overwritten in
//           place, one with another shape is an error.
bool write_group(const std::string &file, const std::string &group, const std::vector<NewDataset> &ds, int mode,
                 std::string &err);

} // namespace h5m

#endif
