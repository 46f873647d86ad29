// PointsDevice.hpp -- the reference's header name; PointsHost and PointsDevice live together in Points.hpp.
#pragma once
#include "CLUEstering/data_structures/Points.hpp"
