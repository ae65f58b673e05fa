/* TEST INFRASTRUCTURE ONLY.  Stand-in for GA's ga-mpi.h: the MPI handle typedefs and
 * constants that TAMM's types.hpp names (single process, never called). */
#pragma once
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Comm;
enum {
  MPI_INT = 1, MPI_C_BOOL, MPI_CHAR, MPI_INT64_T, MPI_UNSIGNED, MPI_UNSIGNED_LONG, MPI_FLOAT,
  MPI_DOUBLE, MPI_COMPLEX, MPI_DOUBLE_COMPLEX, MPI_2INT, MPI_2REAL, MPI_2DOUBLE_PRECISION,
  MPI_MIN, MPI_MAX, MPI_SUM, MPI_MINLOC, MPI_MAXLOC
};
