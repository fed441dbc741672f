// Harness TU for Source/src/General.cu (d_initVoxelArray, d_updateTransforms).
// Test infrastructure.
#include "General.cu"
