/* Type names only; nothing on the hydro pair path performs file I/O. */
#ifndef ORACLE_STUB_HDF5_H
#define ORACLE_STUB_HDF5_H
typedef long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#endif
