// clustering.hpp -- the reference's header name for its host classes, for programs
// written against sg0/nido: everything is in nido_host.hpp (Graph,
// Clustering, GraphGPU, LouvainGPU and the types of types.hpp).
#ifndef NIDO_COMPAT_CLUSTERING_HPP_
#define NIDO_COMPAT_CLUSTERING_HPP_
#include "../nido_host.hpp"
#endif
