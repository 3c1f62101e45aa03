// LvArray's CHAI-managed buffer is a tag here (host memory only); see Array.hpp.
#pragma once
#include "Array.hpp"
