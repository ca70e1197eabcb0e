/* The reference's HDF5 helpers (include/hdf5_util.h, src/hdf5_util.c), same
 * names, arguments and return values (0 on success, negative on failure, a
 * message on stderr), implemented by libgli_b200 without libhdf5 (h5file.cu).
 * Datasets and attributes live in the root group; read_* convert the stored
 * elements to the memory type, write_* store them as mem_type_store. */
#ifndef GLI_B200_COMPAT_HDF5_UTIL_H
#define GLI_B200_COMPAT_HDF5_UTIL_H
#include "hdf5.h"
#include "gli_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

herr_t get_hdf5_dataset_ndims(hid_t file, const char* name, int* ndims);
herr_t get_hdf5_dataset_dims(hid_t file, const char* name, hsize_t* dims);
herr_t read_hdf5_dataset(hid_t file, const char* name, hid_t mem_type, void* data);
herr_t write_hdf5_dataset(hid_t file, const char* name, int degree, const hsize_t dims[], hid_t mem_type_store,
	hid_t mem_type_input, const void* data);
herr_t get_hdf5_attribute_dims(hid_t file, const char* name, hsize_t* dims);
herr_t read_hdf5_attribute(hid_t file, const char* name, hid_t mem_type, void* data);
herr_t write_hdf5_scalar_attribute(hid_t file, const char* name, hid_t mem_type_store, hid_t mem_type_input,
	const void* data);
herr_t write_hdf5_vector_attribute(hid_t file, const char* name, hid_t mem_type_store, hid_t mem_type_input,
	const glong length, const void* data);

#ifdef __cplusplus
}
#endif
#endif
