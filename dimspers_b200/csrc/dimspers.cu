// Single translation unit of the device library: the kernels share their
// __constant__ tables (quadrature, multigrid child maps) without relocatable
// device code.
#include "assemble.cu"
#include "ops.cu"
#include "mg.cu"
#include "mgtail.cu"
#include "solver.cu"
#include "graph.cu"
#include "capi.cu"
#include "stress.cu"
#include "rheology.cu"
#include "fabric.cu"
#include "thermal.cu"
#include "noalloc.cu"
#include "cnn.cu"
