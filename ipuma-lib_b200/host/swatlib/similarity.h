// swatlib substitution tables and matrix selection
// (src/swatlib/similarity.h:9-129, src/swatlib/similarity.cpp).
#ifndef IPUMA_B200_SWATLIB_SIMILARITY_H
#define IPUMA_B200_SWATLIB_SIMILARITY_H

#include <cstdint>
#include <string>
#include <vector>

#include "matrix.h"

namespace swatlib {

// +1 if the characters are equal, -1 otherwise.
int simpleSimilarity(char a, char b);

// 16 x 16 IUPAC compatibility table (1 = compatible), order N A T C G U R Y K M S W B D H V.
extern const std::vector<int8_t> NA_SUBSTITUTION;
// 25 x 25 BLOSUM tables, order A R N D C Q E G H I L K M F P S T W Y V B J Z X *.
// Amino-acid codes 20..24 (B Z X * unknown) index rows B J Z X * (as in the reference).
extern const std::vector<int8_t> BLOSUM50;
extern const std::vector<int8_t> BLOSUM62;

extern const Matrix<int8_t> NA_MATRIX;
extern const Matrix<int8_t> BLOSUM50_MATRIX;
extern const Matrix<int8_t> BLOSUM62_MATRIX;

enum class Similarity { nucleicAcid, blosum50, blosum62, simple };

Similarity strToSimilarity(std::string s);
std::string similarityToStr(Similarity s);

// Maps a 1/0 compatibility matrix to pos/neg and puts `ambig` in row 0 and
// column 0 (the 'N' code).
template <typename T>
Matrix<T> scaleMatrix(Matrix<T> mat, T pos, T neg, T ambig);

// profile(i, j) = scores(sequence[i], j)
Matrix<int8_t> createQueryProfile(const std::vector<uint8_t>& sequence, const Matrix<int8_t>& scores);

template <typename T>
Matrix<T> convertMatrix(const Matrix<int8_t>& om);

// NA: scaled IUPAC table; blosum50/62: the table as is; simple: throws.
Matrix<int8_t> selectMatrix(Similarity s, int8_t matchValue, int8_t mismatchValue, int8_t ambiguityValue);

}  // namespace swatlib
#endif
