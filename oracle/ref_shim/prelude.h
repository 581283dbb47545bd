/* Headers that MKL and Eigen normally pull in transitively for the
 * reference sources; force-included when compiling them. */
#pragma once
#include <omp.h>
#include <functional>
#include <numeric>
#include <cstring>
#include <sstream>
#include <queue>
#include <climits>
#include <unistd.h>
#include <iostream>
#include <format>
