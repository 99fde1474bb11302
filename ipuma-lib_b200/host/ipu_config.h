// Scoring and batching configuration (src/ipu_config.h:1-52).
//
// SWConfig and IPUAlgoConfig keep the reference's fields, order and defaults
// so aggregate initialisation in caller code compiles unchanged.  The
// IPU-only fields of IPUAlgoConfig (vtype, useRemoteBuffer, ioTiles) are
// accepted and ignored; tilesUsed x maxBatches and bufsize still define the
// wire buffer that prepare_remote fills.
#ifndef IPUMA_B200_IPU_CONFIG_H
#define IPUMA_B200_IPU_CONFIG_H

#include <string>

#include "swatlib/swatlib.h"
#include "types.h"

#if defined(__has_include)
#if __has_include(<nlohmann/json.hpp>)
#include <nlohmann/json.hpp>
#define IPUMA_B200_HAVE_NLOHMANN 1
#endif
#endif

namespace ipu {

struct SWConfig {
  int gapInit = 0;
  int gapExtend = -1;
  int matchValue = 1;
  int mismatchValue = -1;
  int ambiguityValue = -1;
  swatlib::Similarity similarity = swatlib::Similarity::nucleicAcid;
  swatlib::DataType datatype = swatlib::DataType::nucleicAcid;
};

struct IPUAlgoConfig {
  int tilesUsed = 1;    // number of buckets (IPU: active vertices)
  int maxAB = 300;      // maximum length of a single sequence A
  int maxBatches = 20;  // maximum number of comparisons per bucket
  int bufsize = 3000;   // bytes of sequence per bucket
  VertexType vtype = VertexType::cpp;
  Algorithm fillAlgo = Algorithm::fillFirst;
  bool forwardOnly = false;  // skip the reverse pass (no start coordinates)
  bool useRemoteBuffer = false;
  int transmissionPrograms = 1;
  int ioTiles = 0;

  int getTotalNumberOfComparisons() const;
  int getBufsize32b() const;
  int getTotalBufsize32b() const;
  int getMetaBufferSize32b() const;
  int getLenBufferSize32b() const;
  int getInputBufferSize32b() const;
};

// Flat JSON text of the configs, with the same keys as the reference's
// to_json (src/ipu_config.cpp:16-80).  to_json(SWConfig) writes the real
// mismatchValue (the reference writes ambiguityValue under that key).
std::string toJsonString(const SWConfig& c);
std::string toJsonString(const IPUAlgoConfig& c);
SWConfig swConfigFromJson(const std::string& text);
IPUAlgoConfig algoConfigFromJson(const std::string& text);

#ifdef IPUMA_B200_HAVE_NLOHMANN
using json = nlohmann::json;
void to_json(json& j, const SWConfig& c);
void from_json(const json& j, SWConfig& c);
void to_json(json& j, const IPUAlgoConfig& c);
void from_json(const json& j, IPUAlgoConfig& c);
#endif

}  // namespace ipu

#endif
