// The 26 neighbour directions in the reference's order (NeighborX / NeighborY / NeighborZ,
// src/CAinitialize.cpp:595-674) and compile-time encodings of them
// for device code. Device code reads a direction's components, its opposite and the capture pass's
// slot order from these immediates with shifts, so that lanes asking for different directions need
// no table in memory.
#pragma once

namespace exaca {

inline constexpr int kNeighborX[26] = {0, 1, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, 0, 1, -1, 0, 0, 1, -1, 1, -1};
inline constexpr int kNeighborY[26] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};
inline constexpr int kNeighborZ[26] = {0, 0, 0, 1, -1, 1, 1, -1, -1, 1, -1, 1, 1, -1, -1, 0, 0, 0, 0, 0, 1, -1, 1, 1, -1, -1};

namespace dirs {

// directions whose component in a table equals v, as a 26-bit mask
constexpr unsigned int with(const int (&t)[26], int v) {
    unsigned int m = 0;
    for (int l = 0; l < 26; l++)
        if (t[l] == v)
            m |= 1u << l;
    return m;
}

// the direction of offset (dz, dx, dy), -1 for none
constexpr int of(int dz, int dx, int dy) {
    for (int l = 0; l < 26; l++)
        if (kNeighborZ[l] == dz && kNeighborX[l] == dx && kNeighborY[l] == dy)
            return l;
    return -1;
}

constexpr int opposite(int l) { return of(-kNeighborZ[l], -kNeighborX[l], -kNeighborY[l]); }

// slot s of the capture pass: the directions ordered by z, then x, then y (consecutive slots are
// neighbours in one row of three cells)
constexpr int slot(int s) {
    int n = 0;
    for (int q = 0; q < 27; q++) {
        const int l = of(q / 9 - 1, (q / 3) % 3 - 1, q % 3 - 1);
        if (l < 0)
            continue;
        if (n == s)
            return l;
        n++;
    }
    return -1;
}

// 5-bit fields i = first .. first + 11 of a 26-entry table f, in one 64-bit word
template <int (*F)(int)> constexpr unsigned long long pack5(int first) {
    unsigned long long w = 0;
    for (int i = first; i < first + 12 && i < 26; i++)
        w |= (unsigned long long)F(i) << (5 * (i - first));
    return w;
}

} // namespace dirs

inline constexpr unsigned int kDirXP = dirs::with(kNeighborX, 1), kDirXM = dirs::with(kNeighborX, -1);
inline constexpr unsigned int kDirYP = dirs::with(kNeighborY, 1), kDirYM = dirs::with(kNeighborY, -1);
inline constexpr unsigned int kDirZP = dirs::with(kNeighborZ, 1), kDirZM = dirs::with(kNeighborZ, -1);
// 5 bits per entry, entries 0-11, 12-23 and 24-25 in three words
inline constexpr unsigned long long kOppA = dirs::pack5<dirs::opposite>(0), kOppB = dirs::pack5<dirs::opposite>(12),
                                    kOppC = dirs::pack5<dirs::opposite>(24);
inline constexpr unsigned long long kSlotA = dirs::pack5<dirs::slot>(0), kSlotB = dirs::pack5<dirs::slot>(12),
                                    kSlotC = dirs::pack5<dirs::slot>(24);

} // namespace exaca
