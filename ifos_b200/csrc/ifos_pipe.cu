// The pipelined stencil launches of one half stencil width FD (IFOS_PIPE_FD,
// set on the command line): the build compiles this file once per FD = 1..6,
// in parallel, and links the objects into libifos_b200.
#ifndef IFOS_PIPE_FD
#error "IFOS_PIPE_FD (1..6) must be defined"
#endif
#include "ifos_launch.cuh"

template void Launcher<float>::v_pipe<IFOS_PIPE_FD>(int, int, int);
template void Launcher<float>::s_pipe<IFOS_PIPE_FD>(int);
