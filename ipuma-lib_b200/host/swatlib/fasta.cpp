#include "fasta.h"

namespace swatlib {

std::istream& operator>>(std::istream& is, Fasta& f) {
  f.description.clear();
  f.sequence.clear();
  std::string line;
  // skip to the header line
  while (is.peek() != EOF && is.peek() != '>') std::getline(is, line);
  if (is.peek() == EOF) {
    is.setstate(std::ios::failbit);
    return is;
  }
  std::getline(is, line);
  f.description = line.substr(1);
  while (is.peek() != EOF && is.peek() != '>') {
    std::getline(is, line);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    f.sequence += line;
  }
  return is;
}

std::vector<Fasta> readFasta(std::istream& is) {
  std::vector<Fasta> out;
  Fasta f;
  while (is >> f) out.push_back(f);
  return out;
}

}  // namespace swatlib
