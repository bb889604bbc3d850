#ifndef REF_HOST_HDF5_SHIM_H
#define REF_HOST_HDF5_SHIM_H
typedef bool hbool_t;
#endif
