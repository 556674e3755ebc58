// k_plane32.cu -- the one-CTA-per-plane transforms of k_plane.cu
// instantiated for the FP32 storage form: float velocity, float2 spectrum
// and float potential (the step's solve), and FP64 source / potential around
// a float2 spectrum (the refined standalone solve).  A separate translation
// unit so that the FP64 and FP32 instantiations compile in parallel.
#define PTC_STORE32 1
#include "k_plane.cu"
