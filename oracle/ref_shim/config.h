/* Build configuration for compiling QUICK's CUDA sources as host code
   (stands in for src/config.h, which QUICK's Makefile copies from
   src/config/config.cuda.h).  DEBUG is left undefined: it only adds timers
   and prints. */
#define CUDA
#undef DEBUG
#undef MPI
