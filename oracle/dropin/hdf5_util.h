/* Stand-in for the reference's include/hdf5_util.h (declarations only; the
 * definitions in hdf5_stub.c all fail).  Test infrastructure for the drop-in
 * build of the reference's python/pymodule.c against libgli_b200. */
#ifndef GLI_DROPIN_HDF5_UTIL_H
#define GLI_DROPIN_HDF5_UTIL_H
#include "hdf5.h"
#include "gli_b200.h"
herr_t get_hdf5_dataset_dims(hid_t file, const char* name, hsize_t* dims);
herr_t read_hdf5_dataset(hid_t file, const char* name, hid_t mem_type, void* data);
herr_t read_hdf5_attribute(hid_t file, const char* name, hid_t mem_type, void* data);
#endif
