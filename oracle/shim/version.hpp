// Oracle test shim for the reference's CMake-generated version header.
#ifndef DMS_SHIM_VERSION_HPP
#define DMS_SHIM_VERSION_HPP
#ifndef DMS_REFERENCE_DIR
#error "DMS_REFERENCE_DIR (the data directory of the reference build) must be defined by the build"
#endif
#define PROJECT_DIR DMS_REFERENCE_DIR
#define PROJECT_NAME "DaMaSCUS-SUN"
#define PROJECT_VERSION "oracle"
#define GIT_BRANCH "none"
#define GIT_COMMIT_HASH "none"
#define DAMASCUS_SUN_LOGO ""
#endif
