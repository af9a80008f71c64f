/*
 * Extra force-include for src/map3d_optimizer.cpp only: line 1035 passes the
 * literal `false` where a `const int*` (null) is expected, which C++11 and
 * later reject.  Spelling `false` as the integer literal 0 inside that unit
 * restores the original meaning (a null pointer there, 0 == false elsewhere).
 * The standard headers are included first so they are unaffected.
 */
#include "ref_compat.h"
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <fstream>
#include <functional>
#include <initializer_list>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <tuple>
#include <utility>
#include <vector>
#include <omp.h>
#define false 0
