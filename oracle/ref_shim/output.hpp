// LvArray's stream output of arrays is not needed by the oracle's reference build.
#pragma once
#include "Array.hpp"
