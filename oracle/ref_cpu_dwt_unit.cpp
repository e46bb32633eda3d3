/*
 * ref_cpu_dwt_unit.cpp — compiles the reference's CPU inverse DWT / MCT
 * (decoder/codec/src/bmi_cpu_dwt_decoder.cpp) from where it lies, by #include, and adds the
 * explicit template instantiations that decoderconcrete.cpp:1623-1783 links against (the
 * reference defines these member templates in the .cpp and never instantiates the int_16 /
 * float forms there).  TEST AND BASELINE INFRASTRUCTURE ONLY (oracle/build_ref_cpu.sh).
 */
#include "bmi_cpu_dwt_decoder.cpp"

namespace BMI {
template void CpuDwtDecoder::VDWT_R53<int_32>(int_32 *, int_32 *, int, int, int, int, int, uint_8, int);
template void CpuDwtDecoder::VDWT_R53<int_16>(int_16 *, int_16 *, int, int, int, int, int, uint_8, int);
template void CpuDwtDecoder::RRct_53<int_32>(void *, int_32 *, int_32 *, int_32 *, int, int, int, int, OutputFormat, int);
template void CpuDwtDecoder::RRct_53<int_16>(void *, int_16 *, int_16 *, int_16 *, int, int, int, int, OutputFormat, int);
template void CpuDwtDecoder::MergeComponents<int_32>(unsigned char *, int_32 *, int_32 *, int_32 *, int_32 *, int, int, int,
                                                     short, OutputFormat, short);
template void CpuDwtDecoder::MergeComponents<float>(unsigned char *, float *, float *, float *, float *, int, int, int, short,
                                                    OutputFormat, short);
}  // namespace BMI
