/*
 * bmi_decoder.h — the reference's public C++ decoder interface, re-declared for this
 * library so existing callers compile and link against it unchanged.
 *
 * Interface being replaced: BMI::Decoder and its configuration / property types in
 * decoder/common/include/codec_base.h:13-345 and codec_datatype.h:15-88, with the
 * singleton entry points Decoder::Get()/Terminate() of decoder/common/src/decoder.cpp:77-92.
 * Names, member order, enum values and status semantics are kept identical (that is what
 * makes it a drop-in); the implementation (src: bmi_decoder.cpp) decodes on the GPU
 * through include/j2k_gpu.h.
 */
#ifndef BMI_DECODER_H
#define BMI_DECODER_H

#include <stdint.h>

typedef int int_32;
typedef unsigned int uint_32;
typedef short int_16;
typedef unsigned short uint_16;
typedef unsigned char uint_8;

typedef enum EncodeMathod_e { Ckernels_W5X3, Ckernels_W9X7, UNKNOWN_MATHOD } EncodeMathod;
typedef enum EncodeFormat_e { RAW, RGB, YUV444, YUV422, YUV420, BAYERGRB, COMPONENT4, UNKNOWN_FORMAT } EncodeFormat;

typedef enum OutputFormat_e {
  IMAGE_FOTMAT_32BITS_ARGB = 0,
  IMAGE_FOTMAT_48BITS_RGB,
  IMAGE_FOTMAT_24BITS_RGB,
  IMAGE_FOTMAT_32BITS_4COMPONENTS,
  IMAGE_FOTMAT_64BITS_4COMPONENTS,
  IMAGE_FOTMAT_48BITS_3COMPONENTS,
  IMAGE_FOTMAT_24BITS_3COMPONENTS,
  IMAGE_FOTMAT_NONE,
  IMAGE_FOTMAT_64BITS_ARGB,
  IMAGE_FOTMAT_36BITS_RGB,
  IMAGE_FOTMAT_48BITS_ARGB
} OutputFormat;

struct ShortSize_s {
  short x;
  short y;
};
typedef struct ShortSize_s sSize, sPos, s2d;

typedef enum enum_dec_progression { UNKNOWN_PROGRESSION = -1, LRCP, RLCP, RPCL, PCRL, CPRL } Jp2_Progression;

#ifdef __cplusplus
namespace BMI {

const int INVALID = -1;

typedef enum Status_e {
  INVALID_STATUS = INVALID,
  READY = 0,
  PARSING,
  PARSE_ERROR,
  PARSE_ERROR_INPUTFILE_ERROR,
  PARSE_ERROR_INVALID_INPUT,
  PARSE_ERROR_UNKNOWN_FORMAT,
  PARSE_ERROR_UNSUPPORTED_FORMAT,
  DECODE_IGNORED,
  DECODING,
  ENCODING = DECODING,
  PRE_DECODE_ERROR,
  PRE_ENCODE_ERROR = PRE_DECODE_ERROR,
  DECODE_ERROR,
  ENCODE_ERROR = DECODE_ERROR,
  RELEASED,
  ENGINE_EXPIRED,
  UNKNOWN
} Status,
    *P_Status;

typedef int CodeStreamHandler;

typedef struct CodeStreamProperties_s {
  sSize mSize;
  sSize mOutputSize;
  sSize mThumbOutputSize;
  OutputFormat mOutputFormat;
  sSize mCodeBlockSize;
  sSize mTileSize;
  s2d mTileNum;
  short mComponentNum;
  short mCalculatedComponentNum;
  short mDwtLevel;
  short mLayer;
  short mBitDepth;
  short mRoiShift;
  EncodeFormat mFormat;
  EncodeMathod mMethod;
  Jp2_Progression mProgression;
  int mHeaderLength;
} CodeStreamProperties, *P_CodeStreamProperties;

typedef enum WordLength_e { USHORT_16_BITS = 2, UINT_32_BITS = 4 } WordLength;

typedef struct EnginConfig_s {
  EnginConfig_s()
      : mInputQueueLen(1), mOutputQueueLen(1), mThreadNum(0), mCpuCoresNum(1), mSyncMode(true), mUsingGpu(true),
        mGpuT1(false) {}
  int mInputQueueLen;
  int mOutputQueueLen;
  int mThreadNum;
  int mCpuCoresNum;
  bool mSyncMode;
  bool mUsingGpu;
  bool mGpuT1;
} EnginConfig, *P_EnginConfig;

typedef struct CodecJobConfig_s {
  CodecJobConfig_s() : mWordLength(UINT_32_BITS), mIgnoreComponents(0) {}
  WordLength mWordLength;
  unsigned int mIgnoreComponents;
} CodecJobConfig, *P_CodecJobConfig;

typedef struct DecodeJobConfig_s : public CodecJobConfig_s {
  DecodeJobConfig_s() : mCheckOutComponent(INVALID), mDwtDecodeTopLevel(-1), mOutputFormat(IMAGE_FOTMAT_NONE) {}
  int mCheckOutComponent;
  int mDwtDecodeTopLevel;
  OutputFormat mOutputFormat;
} DecodeJobConfig, *P_DecodeJobConfig;

class Decoder {
 public:
  virtual CodeStreamHandler Decode(const void *codeStreamBuffer, int bufSize) = 0;
  virtual CodeStreamHandler Decode(const void *codeStreamBuffer, int bufSize, double &time) = 0;
  virtual Status PreDecode(const void *codeStreamBuffer, int bufSize, CodeStreamProperties &properties) = 0;

  static Decoder *Get();
  static void Terminate();

  virtual void GetVersion(int &mainVersion, int &subvVrsion, int &branchVersion, int &year, int &month,
                          int &date) = 0;

  virtual int Init(const P_EnginConfig enginConfig = 0) = 0;
  virtual const EnginConfig *GetEngineConfig() const = 0;

  virtual void SetJobConfig(const DecodeJobConfig &config) = 0;
  virtual void GetJobConfig(DecodeJobConfig &config, CodeStreamHandler handler = INVALID) const = 0;

  virtual Status CheckStatus(CodeStreamHandler handler) const = 0;
  virtual bool CheckProperties(CodeStreamHandler handler, CodeStreamProperties &properties) const = 0;
  virtual const void *GetResult(CodeStreamHandler handler, int &bufSize) = 0;
  virtual const void *GetThumbnail(CodeStreamHandler handler, int &bufSize) = 0;
  virtual const int *GetDecodedComponentInt(CodeStreamHandler handler, int &bufSize, int componentId,
                                            int tileId = INVALID) = 0;
  virtual const float *GetDecodedComponentFloat(CodeStreamHandler handler, int &bufSize, int componentId,
                                                int tileId = INVALID) = 0;
  virtual void Release(CodeStreamHandler handler) = 0;

  virtual ~Decoder() {}
};

}  // namespace BMI
#endif /* __cplusplus */

#endif
