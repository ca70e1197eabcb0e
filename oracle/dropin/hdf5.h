/* Minimal stand-in for <hdf5.h> so that the reference's python/pymodule.c
 * compiles without libhdf5 (test infrastructure for the drop-in check).
 * Every HDF5 call fails, so load_sparse_eri_gausslet_integrals raises
 * RuntimeError; nothing else in the module touches HDF5. */
#ifndef GLI_DROPIN_HDF5_H
#define GLI_DROPIN_HDF5_H
#include <stdint.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#define H5F_ACC_RDONLY 0u
#define H5P_DEFAULT 0
#define H5T_NATIVE_LLONG 0
#define H5T_NATIVE_DOUBLE 1
#define H5T_NATIVE_INT 2
static inline hid_t H5Fopen(const char* name, unsigned flags, hid_t plist) { (void)name; (void)flags; (void)plist; return -1; }
static inline herr_t H5Fclose(hid_t f) { (void)f; return 0; }
#endif
