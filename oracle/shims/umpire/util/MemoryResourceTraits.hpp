// Stand-in: traits header for the umpire shim (test oracle only).
#include <umpire/Umpire.hpp>
