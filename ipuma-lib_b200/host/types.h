// Shared types of the ipuma driver API (src/types.h:1-31).
#ifndef IPUMA_B200_TYPES_H
#define IPUMA_B200_TYPES_H

#include <cstdint>
#include <string>
#include <vector>

#define IPU_JSON_LOG_TAG "IPUSWLOG"

namespace ipu {
typedef std::vector<std::string> RawSequences;
typedef std::vector<uint8_t> EncSequences;

// Index pair into a sequence pool (compare_mn_local).
struct __attribute__((__packed__)) Comparison {
  int32_t indexA;
  int32_t indexB;
};

typedef std::vector<Comparison> Comparisons;

// The four IPU vertex types all compute the same recurrence; on B200 the
// value is accepted and recorded, and selects nothing.
enum class VertexType { cpp, assembly, multi, multiasm };
static const std::vector<std::string> vertexTypeNames = {"cpp", "assembly", "multi", "multiasm"};
enum class Algorithm { fillFirst, roundRobin, greedy };
static const std::vector<std::string> algoNames = {"fillfirst", "roundrobin", "greedy"};

static const std::string typeLabels[] = {"SWAffine", "SWAffineAsm", "MultiSWAffine", "MultiSWAffineAsm"};
std::string vertexTypeToIpuLabel(VertexType v);
std::string vertexTypeToConfigString(VertexType v);
std::string algorithmToConfigString(Algorithm a);
VertexType strToVertexType(std::string s);
Algorithm strToAlgorithm(std::string s);
}  // namespace ipu

#endif
