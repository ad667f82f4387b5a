// utils.hpp -- enums, logging macros and constants of the planc C++ API
// (reference common/utils.h:10-55).
#pragma once
#include <iostream>

#include "mat.hpp"

// common/utils.h:10-11; values are part of the API (the CLI passes -a <int>)
enum algotype { MU, HALS, ANLSBPP, NAIVEANLSBPP, AOADMM, NESTEROV, CPALS, GNSYM, R2, PGD, PGNCG };

#ifndef ERR
#define ERR std::cerr
#endif
#ifndef WARN
#define WARN std::cerr
#endif
#ifndef INFO
#define INFO std::cout
#endif
#ifndef OUTPUT
#define OUTPUT std::cout
#endif

typedef unsigned int UINT;  // common/utils.h:76

// common/utils.h:46-49
#define EPSILON_1EMINUS16 0.00000000000000001
#define EPSILON_1EMINUS8 0.00000001
#define EPSILON 0.000001
#define EPSILON_1EMINUS12 1e-12
