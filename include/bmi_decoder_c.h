/*
 * bmi_decoder_c.h — plain-C surface over the BMI::Decoder singleton (include/bmi_decoder.h)
 * for FFI callers (ctypes, cgo, JNI, N-API) that cannot call C++ virtual functions.
 *
 * There is no counterpart file in the reference; each function forwards to one method of
 * the reference's C++ interface (decoder/common/include/codec_base.h:316-345) with the
 * same argument meaning and the same status values (BMI::Status as int).
 */
#ifndef BMI_DECODER_C_H
#define BMI_DECODER_C_H

#ifdef __cplusplus
extern "C" {
#endif

/* Decoder::Get()->Init() with mSyncMode / mOutputQueueLen set; 0 = ok. */
int bmi_decoder_init(int sync_mode, int output_queue_len);
/* Decoder::SetJobConfig(): mOutputFormat, mDwtDecodeTopLevel, mIgnoreComponents, mCheckOutComponent. */
void bmi_decoder_set_job(int output_format, int dwt_top_level, unsigned ignore_components, int checkout_component);
/* Decoder::Decode(buf, size, time): returns the handler; *ms receives the time. */
int bmi_decoder_decode(const void *buf, int size, double *ms);
/* Decoder::PreDecode(): returns a BMI::Status, fills the main-header properties. */
int bmi_decoder_predecode(const void *buf, int size, int *width, int *height, int *ncomp, int *bitdepth, int *levels);
/* Decoder::PreDecode() as above, reporting CodeStreamProperties::mFormat (EncodeFormat: RAW,
 * RGB, YUV444, YUV422, YUV420, BAYERGRB, COMPONENT4; from the component sampling and the
 * JP2 colour space, dec_jp2.cpp:488-523) and mMethod (0 = 5/3, 1 = 9/7).  Host only. */
int bmi_decoder_predecode_format(const void *buf, int size, int *format, int *method);
/* Decoder::CheckStatus() */
int bmi_decoder_status(int handler);
/* Decoder::GetResult() / GetThumbnail() / GetDecodedComponentInt() / GetDecodedComponentFloat() */
const void *bmi_decoder_result(int handler, int *size);
const void *bmi_decoder_thumbnail(int handler, int *size);
const int *bmi_decoder_component_int(int handler, int component, int *size);
const float *bmi_decoder_component_float(int handler, int component, int *size);
/* Decoder::Release() and Decoder::Terminate() */
void bmi_decoder_release(int handler);
void bmi_decoder_terminate(void);

#ifdef __cplusplus
}
#endif
#endif
