/* Empty stand-in for <hdf5.h>.  The reference's io.h includes HDF5 only for
 * its HDF5 writer (src/io.c:132-301), which the oracle build does not compile;
 * mc_cpu.c and mc_gpu.cu need io.h solely for <stdio.h>/<string.h>.  This
 * file lets those sources compile unmodified without an HDF5 installation. */
