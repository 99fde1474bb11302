#include "ipu_config.h"

#include <cctype>
#include <map>
#include <sstream>
#include <stdexcept>

namespace ipu {

int IPUAlgoConfig::getBufsize32b() const { return (bufsize + 3) / 4; }
int IPUAlgoConfig::getTotalNumberOfComparisons() const { return tilesUsed * maxBatches; }
int IPUAlgoConfig::getMetaBufferSize32b() const { return getTotalNumberOfComparisons() * 4; }
int IPUAlgoConfig::getTotalBufsize32b() const { return tilesUsed * getBufsize32b(); }
int IPUAlgoConfig::getLenBufferSize32b() const { return getTotalNumberOfComparisons(); }
int IPUAlgoConfig::getInputBufferSize32b() const { return getTotalBufsize32b() + getMetaBufferSize32b(); }

namespace {

// Minimal parser for a flat JSON object of numbers, strings and booleans.
std::map<std::string, std::string> parseFlat(const std::string& t) {
  std::map<std::string, std::string> out;
  size_t i = 0;
  auto ws = [&] {
    while (i < t.size() && std::isspace(static_cast<unsigned char>(t[i]))) ++i;
  };
  auto str = [&]() -> std::string {
    if (t[i] != '"') throw std::runtime_error("json: expected string");
    std::string s;
    for (++i; i < t.size() && t[i] != '"'; ++i) s += t[i];
    ++i;
    return s;
  };
  ws();
  if (i >= t.size() || t[i] != '{') throw std::runtime_error("json: expected object");
  ++i;
  while (true) {
    ws();
    if (i < t.size() && t[i] == '}') break;
    std::string k = str();
    ws();
    if (t[i] != ':') throw std::runtime_error("json: expected ':'");
    ++i;
    ws();
    std::string v;
    if (t[i] == '"') {
      v = str();
    } else {
      while (i < t.size() && t[i] != ',' && t[i] != '}' && !std::isspace(static_cast<unsigned char>(t[i]))) v += t[i++];
    }
    out[k] = v;
    ws();
    if (i < t.size() && t[i] == ',') ++i;
  }
  return out;
}

const std::string& need(const std::map<std::string, std::string>& m, const char* k) {
  auto it = m.find(k);
  if (it == m.end()) throw std::runtime_error(std::string("json: missing key ") + k);
  return it->second;
}

bool asBool(const std::string& v) { return v == "true" || v == "1"; }

}  // namespace

std::string toJsonString(const SWConfig& c) {
  std::ostringstream ss;
  ss << "{\"gapInit\":" << c.gapInit << ",\"gapExtend\":" << c.gapExtend << ",\"matchValue\":" << c.matchValue
     << ",\"mismatchValue\":" << c.mismatchValue << ",\"ambiguityValue\":" << c.ambiguityValue
     << ",\"similarity\":\"" << swatlib::similarityToStr(c.similarity) << "\",\"datatype\":\""
     << swatlib::dataTypeToStr(c.datatype) << "\"}";
  return ss.str();
}

std::string toJsonString(const IPUAlgoConfig& c) {
  std::ostringstream ss;
  ss << "{\"tilesUsed\":" << c.tilesUsed << ",\"maxAB\":" << c.maxAB << ",\"maxBatches\":" << c.maxBatches
     << ",\"bufsize\":" << c.bufsize << ",\"vtype\":\"" << vertexTypeToConfigString(c.vtype)
     << "\",\"fillAlgo\":\"" << algorithmToConfigString(c.fillAlgo) << "\",\"forwardOnly\":"
     << (c.forwardOnly ? "true" : "false") << ",\"useRemoteBuffer\":" << (c.useRemoteBuffer ? "true" : "false")
     << ",\"transmissionPrograms\":" << c.transmissionPrograms << ",\"ioTiles\":" << c.ioTiles << "}";
  return ss.str();
}

SWConfig swConfigFromJson(const std::string& text) {
  auto m = parseFlat(text);
  SWConfig c;
  c.gapInit = std::stoi(need(m, "gapInit"));
  c.gapExtend = std::stoi(need(m, "gapExtend"));
  c.matchValue = std::stoi(need(m, "matchValue"));
  c.mismatchValue = std::stoi(need(m, "mismatchValue"));
  c.ambiguityValue = std::stoi(need(m, "ambiguityValue"));
  c.similarity = swatlib::strToSimilarity(need(m, "similarity"));
  c.datatype = swatlib::strToDataType(need(m, "datatype"));
  return c;
}

IPUAlgoConfig algoConfigFromJson(const std::string& text) {
  auto m = parseFlat(text);
  IPUAlgoConfig c;
  c.tilesUsed = std::stoi(need(m, "tilesUsed"));
  c.maxAB = std::stoi(need(m, "maxAB"));
  c.maxBatches = std::stoi(need(m, "maxBatches"));
  c.bufsize = std::stoi(need(m, "bufsize"));
  c.vtype = strToVertexType(need(m, "vtype"));
  c.fillAlgo = strToAlgorithm(need(m, "fillAlgo"));
  c.forwardOnly = asBool(need(m, "forwardOnly"));
  c.useRemoteBuffer = asBool(need(m, "useRemoteBuffer"));
  c.transmissionPrograms = std::stoi(need(m, "transmissionPrograms"));
  c.ioTiles = std::stoi(need(m, "ioTiles"));
  return c;
}

#ifdef IPUMA_B200_HAVE_NLOHMANN
void to_json(json& j, const SWConfig& c) { j = json::parse(toJsonString(c)); }
void from_json(const json& j, SWConfig& c) { c = swConfigFromJson(j.dump()); }
void to_json(json& j, const IPUAlgoConfig& c) { j = json::parse(toJsonString(c)); }
void from_json(const json& j, IPUAlgoConfig& c) { c = algoConfigFromJson(j.dump()); }
#endif

}  // namespace ipu
