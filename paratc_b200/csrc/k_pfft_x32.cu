// k_pfft_x32.cu -- the x transforms of k_pfft_x.cu instantiated for the
// FP32 storage form: float2 spectra, float velocity and potential (the
// step's solve), and FP64 source / potential around a float2 spectrum (the
// refined standalone solve).  A separate translation unit so that the FP64
// and FP32 instantiations compile in parallel.
#define PTC_STORE32 1
#include "k_pfft_x.cu"
