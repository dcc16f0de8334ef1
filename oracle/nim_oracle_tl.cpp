// Tangent-linear build of the CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// The oracle's source with every computed value a dual number
// (oracle/nim_dual.h): a run gives the FP64 oracle's values bit for bit and
// their derivatives along one seeded direction of nu, alpha and the
// initial/boundary fields, the FP64 tangent-linear reference gradient of the
// hot-wall Nusselt number.  Entry points nim_oracle_tl_* (same arguments as
// nim_oracle_*, plus the seeding and tangent calls at the end of
// nim_oracle.cpp).
#define NIM_ORACLE_TANGENT 1
#include "nim_oracle.cpp"
