// Geometry.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's WKT geometry header, which
// the hot path names only in the declarations of geometric mesh selections.
#pragma once
#include "Config.hpp"
class Point;
class Geometry;
