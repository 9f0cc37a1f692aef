// Test infrastructure (oracle). Force-included (-include) into the reference's own unit tests when
// oracle/Makefile builds them: their CMake build bakes the source tree and a scratch directory into
// the binaries (CUDAEE_SOURCE_DIR, CUDAEE_*TEST_TMP_DIR); here those macros expand to these calls,
// so the binaries run on a host without the reference tree. The fixture files they read are copied
// next to them at build time (_ref/refdata/tests/data).
#ifndef CEE_REF_UNIT_PATHS_H
#define CEE_REF_UNIT_PATHS_H

#include <cstdlib>
#include <filesystem>
#include <string>

// $CEE_REF_UNIT_DATA, else the refdata directory beside the running binary.
inline std::string cee_ref_unit_source_dir() {
  if (const char* env = std::getenv("CEE_REF_UNIT_DATA")) return env;
  return (std::filesystem::read_symlink("/proc/self/exe").parent_path() / "refdata").string();
}

// $CEE_REF_UNIT_TMP, else a directory under the system temporary directory.
inline std::string cee_ref_unit_tmp_dir() {
  if (const char* env = std::getenv("CEE_REF_UNIT_TMP")) return env;
  return (std::filesystem::temp_directory_path() / "cee_ref_unit").string();
}

#endif
