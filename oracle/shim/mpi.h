/* Empty stand-in for <mpi.h>. ORACLE-ONLY TEST INFRASTRUCTURE: NetFlux
   includes <mpi.h> (Includes.hpp:19, parallelization/MPI.hpp:2) but calls no
   MPI function on the solver path, and no MPI implementation is installed. */
#pragma once
