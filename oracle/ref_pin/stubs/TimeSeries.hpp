// TimeSeries.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's boundary time-series
// database; the pin driver sets the boundary value fields directly.
#pragma once
#include "Config.hpp"
#include "DataArray.hpp"
#include "TimeParameters.hpp"
template <typename TT, typename T>
class TimeSeries;
template <typename TT, typename T>
class TimeSeriesDatabase;
