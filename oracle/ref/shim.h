/* Forced-include shim for compiling ProtoMol 2.1 sources with a current g++
 * (test infrastructure: the oracle build only).  The reference defines
 * Constant::M_PI etc. (base/pmconstants.h:40-42), which collide with the
 * libc macros; it also uses two MSVC/autoconf names. */
#include <cmath>
#include <math.h>
#undef M_PI
#undef M_E
#undef M_2_SQRTPI
#undef M_SQRT2
#include <cstring>
#include <cstdlib>
#include <climits>
#include <algorithm>
#include <iostream>
#include <fstream>
#include <sstream>
#define sprintf_s snprintf
#define SOCKLEN_TYPE socklen_t
#include <sys/socket.h>
