// Stand-in for the APComp header included by dray.cpp; only the MPI
// communicator hook is referenced and the oracle is built without MPI.
#ifndef ORACLE_SHIM_APCOMP_HPP
#define ORACLE_SHIM_APCOMP_HPP
namespace apcomp { inline void mpi_comm (int) {} }
#endif
