/*
 * HDF5 stand-in used ONLY to compile the reference PIC3D sources into the
 * CPU oracle.  The reference headers (include/io_utils.h, include/simulation.h)
 * name hid_t and H5P_DEFAULT; the oracle harness replaces the HDF5 writers
 * (src/io_utils.cpp) with raw binary dumps, so nothing else is needed.
 */
#ifndef PIC3D_ORACLE_HDF5_STUB_H
#define PIC3D_ORACLE_HDF5_STUB_H
typedef long hid_t;
typedef int herr_t;
#define H5P_DEFAULT 0
static inline herr_t H5open(void) { return 0; }
static inline herr_t H5close(void) { return 0; }
#endif
