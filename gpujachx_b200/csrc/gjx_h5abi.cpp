// gjx_h5abi.cpp -- C ABI over h5mini (include/gjx.h): read one dataset, write
// a group of datasets.  Errors leave their text in gjx_last_error().
#include <string>
#include <vector>

#include "gjx.h"
#include "gjx_internal.h"
#include "h5mini.h"

extern "C" {

int gjx_h5_read(const char *const file, const char *const path, const int as_float, void *const out,
                const unsigned long long cap, unsigned long long *const dims, int *const rank)
{
  if (!file || !path) {
    gjx::set_error("gjx_h5_read: file and path are required");
    return -1;
  }
  h5m::Array a;
  std::string err;
  if (!h5m::read(file, path, a, err)) {
    gjx::set_error(("gjx_h5_read: " + err).c_str());
    return -2;
  }
  if (a.dims.size() > 8u) {
    gjx::set_error("gjx_h5_read: rank above 8");
    return -3;
  }
  if (rank)
    *rank = (int)a.dims.size();
  if (dims)
    for (size_t i = 0u; i < a.dims.size(); ++i)
      dims[i] = a.dims[i];
  if (!out)
    return 0;
  if (a.count() > cap) {
    gjx::set_error("gjx_h5_read: buffer too small");
    return -4;
  }
  if (as_float) {
    std::vector<double> v;
    a.to_double(v);
    std::copy(v.begin(), v.end(), static_cast<double *>(out));
  }
  else {
    std::vector<int> v;
    if (!a.to_int(v)) {
      gjx::set_error("gjx_h5_read: not an integer dataset");
      return -5;
    }
    std::copy(v.begin(), v.end(), static_cast<int *>(out));
  }
  return 0;
}

int gjx_h5_write(const char *const file, const char *const group, const int mode, const int nds,
                 const char *const *const names, const int *const ranks, const unsigned long long *const dims,
                 const int *const is_float, const void *const *const data)
{
  if (!file || !group || nds < 0 || (nds && (!names || !ranks || !dims || !is_float || !data)) || mode < 0 ||
      mode > 2) {
    gjx::set_error("gjx_h5_write: bad arguments");
    return -1;
  }
  std::vector<h5m::NewDataset> ds((size_t)nds);
  for (int i = 0; i < nds; ++i) {
    if (ranks[i] < 0 || ranks[i] > 8 || !names[i]) {
      gjx::set_error("gjx_h5_write: bad dataset");
      return -1;
    }
    ds[i].name = names[i];
    ds[i].dims.assign(dims + 8 * i, dims + 8 * i + ranks[i]);
    ds[i].is_float = is_float[i] != 0;
    ds[i].data = data[i];
  }
  std::string err;
  if (!h5m::write_group(file, group, ds, mode, err)) {
    gjx::set_error(("gjx_h5_write: " + err).c_str());
    return -2;
  }
  return 0;
}

} // extern "C"
