// Stand-in for APComp's image compositor header.  Devil Ray uses its
// Compositor only across MPI ranks (rendering/renderer.cpp:366-420, under
// DRAY_MPI_ENABLED); the oracle is built without MPI, so nothing of it is
// needed beyond the include.
#ifndef ORACLE_SHIM_APCOMP_COMPOSITOR_HPP
#define ORACLE_SHIM_APCOMP_COMPOSITOR_HPP
#include "apcomp.hpp"
#endif
