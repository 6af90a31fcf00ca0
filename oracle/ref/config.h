/* Hand-written platform configuration for compiling the ProteinDF reference
 * sources directly with g++ (test infrastructure only; the oracle never ships).
 * It states the facts the reference's own configure step would detect on this
 * Linux/glibc image. No BLAS/LAPACK, MPI, Eigen, ViennaCL, HDF5 or libcint. */
#define PROJECT_VERSION "reference-oracle"
#define PROJECT_VERSION_BUILD "reference-oracle"
#define HAVE_SYS_RESOURCE_H
#define HAVE_SYS_TIME_H
#define HAVE_SYS_TYPES_H
#define HAVE_UNISTD_H
#define HAVE_STDINT_H
#define HAVE_LAPACK
#define HAVE_BLAS
#define __restrict__ __restrict
