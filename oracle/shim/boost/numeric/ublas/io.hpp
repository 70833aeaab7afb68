// Stand-in for boost/numeric/ublas/io.hpp. The CTBB_ICD reference includes it
// but streams no uBLAS containers, so it only needs to exist (oracle build).
#pragma once
#include <iostream>
