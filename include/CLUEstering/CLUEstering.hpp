// CLUEstering.hpp -- umbrella header of the clue:: C++ API over libclue_b200
// (the reference's include/CLUEstering/CLUEstering.hpp).  Link with -lclue_b200.
#pragma once

#include "CLUEstering/core/Clusterer.hpp"
#include "CLUEstering/core/ConvolutionalKernel.hpp"
#include "CLUEstering/core/DistanceMetrics.hpp"
#include "CLUEstering/data_structures/AssociationMap.hpp"
#include "CLUEstering/data_structures/ClusterProperties.hpp"
#include "CLUEstering/data_structures/Points.hpp"
#include "CLUEstering/detail/Runtime.hpp"
#include "CLUEstering/utils/cluster_centroid.hpp"
#include "CLUEstering/utils/get_clusters.hpp"
#include "CLUEstering/utils/read_csv.hpp"
#include "CLUEstering/utils/scores.hpp"
#include "CLUEstering/utils/validation.hpp"
