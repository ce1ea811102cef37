/* Forced-include header for compiling ProtoMol 2.1 sources with a current
 * g++ (the drop-in build links ProtoMol's own framework objects).  ProtoMol
 * defines Constant::M_PI etc. (base/pmconstants.h:40-42), which collide with
 * the libc macros, and uses two MSVC / autoconf names. */
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
#define PACKAGE_BUGREPORT "n/a"
#define PACKAGE_HOMEPAGE "n/a"
#define PACKAGE_NAME "ProtoMol"
#define PACKAGE_VERSION "2.1"
#define PACKAGE_STRING "ProtoMol 2.1"
#define VERSION "2.1"
#define PACKAGE "protomol"
#define PACKAGE_CITE "n/a"
#define PACKAGE_WHOAMI "n/a"
#define PACKAGE_UNAME "n/a"
#define PACKAGE_COMPILER "g++"
#define PACKAGE_COMPILER_VERSION "n/a"
#define PACKAGE_COMPILER_OPTIONS "n/a"
#define PACKAGE_PLATFORM "n/a"
#define PACKAGE_DATE "n/a"
