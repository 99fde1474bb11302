// FASTA records and reader (src/swatlib/fasta.h, src/swatlib/fasta.cpp:15-51).
#ifndef IPUMA_B200_SWATLIB_FASTA_H
#define IPUMA_B200_SWATLIB_FASTA_H
#include <istream>
#include <string>
#include <vector>

namespace swatlib {
struct Fasta {
  std::string description;
  std::string sequence;
};
// Reads one record; false at end of input (a record read up to EOF is kept).
std::istream& operator>>(std::istream& is, Fasta& f);
std::vector<Fasta> readFasta(std::istream& is);
}  // namespace swatlib
#endif
