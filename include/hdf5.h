/* The part of the HDF5 C interface that the reference's code uses for its
 * files (python/pymodule.c:1181-1331, cli/gli_eri_integrals.c:40-163, through
 * src/hdf5_util.c), served by libgli_b200 without libhdf5: the handle and size
 * types, the file open / create / close calls (mapped onto gli_b200_h5_*), and
 * the type ids of the stored and in-memory elements.  Files read and written
 * this way are ordinary HDF5 files (superblock version 0, symbol-table
 * groups, contiguous datasets, version-1 attributes); see h5file.cu.
 *
 * This header replaces <hdf5.h> only for code compiled against include/ and
 * linked to libgli_b200 (the reference's CLI and Python module); nothing of
 * libhdf5 is declared beyond these names. */
#ifndef GLI_B200_HDF5_H
#define GLI_B200_HDF5_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5F_ACC_RDONLY 0x0000u
#define H5F_ACC_RDWR 0x0001u
#define H5F_ACC_TRUNC 0x0002u
#define H5P_DEFAULT ((hid_t)0)

/* element types: in memory (NATIVE) and as stored (little-endian) */
#define H5T_NATIVE_DOUBLE ((hid_t)0x7f000001)
#define H5T_NATIVE_LLONG ((hid_t)0x7f000002)
#define H5T_NATIVE_INT ((hid_t)0x7f000003)
#define H5T_IEEE_F64LE ((hid_t)0x7f000011)
#define H5T_STD_I64LE ((hid_t)0x7f000012)
#define H5T_STD_I32LE ((hid_t)0x7f000013)

/* open an existing file (the whole file is parsed here; -1 when it is not a
 * readable HDF5 file of this subset) */
hid_t gli_b200_h5_fopen(const char* name, unsigned flags, hid_t fapl);
/* create (truncate) a file; its contents are written by gli_b200_h5_fclose */
hid_t gli_b200_h5_fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t gli_b200_h5_fclose(hid_t file);

#define H5Fopen gli_b200_h5_fopen
#define H5Fcreate gli_b200_h5_fcreate
#define H5Fclose gli_b200_h5_fclose

#ifdef __cplusplus
}
#endif
#endif
