// Output files in the reference's binary format (outputFileType 101).
//
// writeBinaryFile (src/io/binary_io.cc:185-216) writes the raw bytes of one
// Quantities vector -- cells x components floats, native byte order, no
// header -- to one file per field; writeOutputData
// (src/input_output.cc:216-275) names the files after the output name plus a
// suffix per field (".den", ".vel", ... for uQuantities, ".a_den", ... for
// aQuantities).  The reference writes at most 256^3 elements per call to
// ostream::write; here one file write per chunk of a few MB gives the same
// bytes.

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/dtfe_host.h"

namespace {

// src/input_output.cc:224-274, in field-slot order
const char* const kSuffix[DTFE_NUM_FIELDS] = {".den",      ".vel",     ".velGrad", ".velDiv",    ".velShear",
                                              ".velVort",  nullptr,    ".scalar",  ".scalarGrad"};
const char* const kSuffixAveraged[DTFE_NUM_FIELDS] = {".a_den",      ".a_vel",     ".a_velGrad",
                                                      ".a_velDiv",   ".a_velShear", ".a_velVort",
                                                      ".a_velStd",   ".a_scalar",  ".a_scalarGrad"};

}  // namespace

extern "C" {

const char* dtfe_field_suffix(int32_t slot, int32_t averaged) {
  if (slot < 0 || slot >= DTFE_NUM_FIELDS) return nullptr;
  return averaged ? kSuffixAveraged[slot] : kSuffix[slot];
}

int dtfe_write_binary(const char* path, const void* data, int64_t bytes) {
  if (!path || bytes < 0 || (bytes > 0 && !data)) return DTFE_ERR_ARG;
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return DTFE_ERR_IO;
  const char* p = static_cast<const char*>(data);
  const int64_t chunk = int64_t(1) << 24;
  int rc = DTFE_OK;
  for (int64_t at = 0; at < bytes && rc == DTFE_OK; at += chunk) {
    const size_t n = (size_t)(bytes - at < chunk ? bytes - at : chunk);
    if (std::fwrite(p + at, 1, n, f) != n) rc = DTFE_ERR_IO;
  }
  if (std::fclose(f) != 0 && rc == DTFE_OK) rc = DTFE_ERR_IO;
  return rc;
}

}  // extern "C"
