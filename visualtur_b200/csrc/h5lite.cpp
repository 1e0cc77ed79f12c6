/*
 * h5lite.cpp -- minimal HDF5 container support for one contiguous 3-D
 * dataset.
 */
#include "vt_runtime.h"

namespace vtrt {
bool h5_locate(const unsigned char*, size_t, const char*, int*, int64_t*, uint64_t*, std::string* why) {
    *why = "HDF5 reader not built";
    return false;
}
bool h5_write(const char*, const char*, const void*, int, const int64_t*, std::string* why) {
    *why = "HDF5 writer not built";
    return false;
}
}  // namespace vtrt
