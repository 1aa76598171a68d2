// Stand-in: QuickPool strategy tag for the umpire shim (test oracle only).
#ifndef ORACLE_SHIM_UMPIRE_QUICKPOOL_HPP
#define ORACLE_SHIM_UMPIRE_QUICKPOOL_HPP
#include <umpire/Umpire.hpp>
namespace umpire { namespace strategy { struct QuickPool {}; } }
#endif
