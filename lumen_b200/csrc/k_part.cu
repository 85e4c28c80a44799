// One part of the engine's kernel instantiations (LUMEN_PART, 0 .. LUMEN_N_PARTS - 1), compiled in parallel with
// the others; lumen_b200.cu declares each launcher extern.
#include "engine.cuh"

#ifndef LUMEN_PART
#error "compile with -DLUMEN_PART=k"
#endif
#define LUMEN_INST_SHAPE(G, B, M, T, A, N) template LUMEN_SHAPE_DECL(G, B, M, T, A, N)
#if LUMEN_PART == 0
LUMEN_SHAPES_0(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 1
LUMEN_SHAPES_1(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 2
LUMEN_SHAPES_2(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 3
LUMEN_SHAPES_3(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 4
LUMEN_SHAPES_4(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 5
LUMEN_SHAPES_5(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 6
LUMEN_SHAPES_6(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 7
LUMEN_SHAPES_7(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 8
LUMEN_SHAPES_8(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 9
LUMEN_SHAPES_9(LUMEN_INST_SHAPE)
#elif LUMEN_PART == 10
// the drain's persistent loops are the other parts' instantiations
#define LUMEN_EXTERN_SHAPE(G, B, M, T, A, N) extern template LUMEN_SHAPE_DECL(G, B, M, T, A, N)
LUMEN_SHAPES(LUMEN_EXTERN_SHAPE)
template int run_wave<0>(const Launch&, const Pick&, unsigned long long*, cudaStream_t, int, int, int, float*);
template int run_wave<LUMEN_MAX_GRAD>(const Launch&, const Pick&, unsigned long long*, cudaStream_t, int, int, int,
                                      float*);
#elif LUMEN_PART == 11
template int launch_event_locate<0>(const DScene&, const LumenSource&, int32_t*, cudaStream_t);
template int launch_event_locate<1>(const DScene&, const LumenSource&, int32_t*, cudaStream_t);
template int launch_photons<0>(const Launch&, int32_t*, float*, cudaStream_t);
template int launch_photons<1>(const Launch&, int32_t*, float*, cudaStream_t);
template int launch_query<float>(const DScene&, const float*, const int32_t*, const int32_t*, float, int64_t, int32_t*,
                                 float*, cudaStream_t);
template int launch_query<double>(const DScene&, const double*, const int32_t*, const int32_t*, double, int64_t,
                                  int32_t*, double*, cudaStream_t);
template int launch_locate<float>(const DScene&, const float*, int64_t, int32_t*, cudaStream_t);
template int launch_locate<double>(const DScene&, const double*, int64_t, int32_t*, cudaStream_t);
#endif
