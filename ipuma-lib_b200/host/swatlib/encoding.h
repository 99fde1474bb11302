// swatlib encoders: char -> integer code tables of the reference
// (src/swatlib/encoding.h:12-106, src/swatlib/encoding.cpp).  The code
// assignment is the reference's, so encoded buffers are interchangeable.
#ifndef IPUMA_B200_SWATLIB_ENCODING_H
#define IPUMA_B200_SWATLIB_ENCODING_H

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace swatlib {

enum class DataType { nucleicAcid, aminoAcid, string };

DataType strToDataType(std::string s);
std::string dataTypeToStr(DataType d);

// Nucleic-acid codes: N A T C G U R Y K M S W B D H V, '\0' (unknown) = 16.
extern const std::map<char, uint8_t> NA_CODE;
// Amino-acid codes: A R N D C Q E G H I L K M F P S T W Y V B Z X *, '\0' = 24.
extern const std::map<char, uint8_t> AA_CODE;

class Encoding {
  std::map<char, uint8_t> code;
  std::vector<uint8_t> codeTable;  // 127 entries, default = code of '\0'
  std::vector<char> decodeTable;

 public:
  explicit Encoding(std::map<char, uint8_t> mapping);
  uint8_t encode(char c) const;
  std::vector<uint8_t> encode(const std::string& s) const;
  std::vector<std::vector<uint8_t>> encode(const std::vector<std::string>& ss) const;
  char decode(uint8_t i) const;
  std::string decode(const std::vector<uint8_t>& v) const;
  std::vector<std::string> decode(const std::vector<std::vector<uint8_t>>& vv) const;
  uint8_t get_terminator() const;
  std::vector<uint8_t> getCodeTable() const;
};

class NAEncoding : public Encoding {
 public:
  NAEncoding();
};
class AAEncoding : public Encoding {
 public:
  AAEncoding();
};
class CharEncoding : public Encoding {
 public:
  CharEncoding();
};

Encoding getEncoder(DataType t);

}  // namespace swatlib
#endif
