#include "encoding.h"

#include <cctype>
#include <stdexcept>

namespace swatlib {

const std::map<char, uint8_t> NA_CODE = {
    {'N', 0},  {'A', 1},  {'T', 2},  {'C', 3},  {'G', 4},  {'U', 5},  {'R', 6},  {'Y', 7},  {'K', 8},
    {'M', 9},  {'S', 10}, {'W', 11}, {'B', 12}, {'D', 13}, {'H', 14}, {'V', 15}, {'\0', 16},
};

const std::map<char, uint8_t> AA_CODE = {
    {'A', 0},  {'R', 1},  {'N', 2},  {'D', 3},  {'C', 4},  {'Q', 5},  {'E', 6},
    {'G', 7},  {'H', 8},  {'I', 9},  {'L', 10}, {'K', 11}, {'M', 12}, {'F', 13},
    {'P', 14}, {'S', 15}, {'T', 16}, {'W', 17}, {'Y', 18}, {'V', 19}, {'B', 20},
    {'Z', 21}, {'X', 22}, {'*', 23}, {'\0', 24},
};

DataType strToDataType(std::string s) {
  if (s == "na") return DataType::nucleicAcid;
  if (s == "aa") return DataType::aminoAcid;
  if (s == "str") return DataType::string;
  throw std::runtime_error("Invalid dataType: " + s);
}

std::string dataTypeToStr(DataType d) {
  switch (d) {
    case DataType::aminoAcid: return "aa";
    case DataType::nucleicAcid: return "na";
    case DataType::string: return "str";
  }
  throw std::runtime_error("Invalid DataType");
}

Encoding::Encoding(std::map<char, uint8_t> mapping) : code(std::move(mapping)) {
  const uint8_t term = code.count('\0') ? code.at('\0') : 0;
  codeTable.assign(127, term);
  decodeTable.assign(256, '\0');
  for (const auto& kv : code) {
    const unsigned char key = static_cast<unsigned char>(kv.first);
    if (key < 127) {
      codeTable[key] = kv.second;
      codeTable[static_cast<unsigned char>(std::tolower(key))] = kv.second;
    }
    decodeTable[kv.second] = kv.first;
  }
}

uint8_t Encoding::encode(char c) const {
  const unsigned char u = static_cast<unsigned char>(c);
  return u < 127 ? codeTable[u] : codeTable[0];
}

std::vector<uint8_t> Encoding::encode(const std::string& s) const {
  std::vector<uint8_t> v(s.size());
  for (size_t i = 0; i < s.size(); ++i) v[i] = encode(s[i]);
  return v;
}

std::vector<std::vector<uint8_t>> Encoding::encode(const std::vector<std::string>& ss) const {
  std::vector<std::vector<uint8_t>> vv(ss.size());
  for (size_t i = 0; i < ss.size(); ++i) vv[i] = encode(ss[i]);
  return vv;
}

char Encoding::decode(uint8_t i) const { return decodeTable[i]; }

std::string Encoding::decode(const std::vector<uint8_t>& v) const {
  std::string s(v.size(), ' ');
  for (size_t i = 0; i < v.size(); ++i) s[i] = decode(v[i]);
  return s;
}

std::vector<std::string> Encoding::decode(const std::vector<std::vector<uint8_t>>& vv) const {
  std::vector<std::string> ss(vv.size());
  for (size_t i = 0; i < vv.size(); ++i) ss[i] = decode(vv[i]);
  return ss;
}

uint8_t Encoding::get_terminator() const { return code.count('\0') ? code.at('\0') : 0; }

std::vector<uint8_t> Encoding::getCodeTable() const { return codeTable; }

NAEncoding::NAEncoding() : Encoding(NA_CODE) {}
AAEncoding::AAEncoding() : Encoding(AA_CODE) {}

static std::map<char, uint8_t> charCode() {
  std::map<char, uint8_t> m;
  for (int i = 0; i < 256; ++i) m[static_cast<char>(i)] = static_cast<uint8_t>(i);
  return m;
}
CharEncoding::CharEncoding() : Encoding(charCode()) {}

Encoding getEncoder(DataType t) {
  switch (t) {
    case DataType::aminoAcid: return AAEncoding();
    case DataType::nucleicAcid: return NAEncoding();
    case DataType::string: return CharEncoding();
  }
  throw std::runtime_error("Invalid DataType");
}

}  // namespace swatlib
