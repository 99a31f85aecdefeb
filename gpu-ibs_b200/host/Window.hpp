// One output row of the window scan, as the reference declares it
// (src/Window.hpp:7-16): the contig id, the window's [start, end) and its
// statistics. addVariationOriginal is the reference's gap-to-distance rule
// (src/Window.hpp:29-36); the device computes the same values, this copy
// serves host-side callers that accumulate rows themselves.
#pragma once

#include <cstdlib>
#include <string>

class Window
{
public:
    std::string id;
    int start = 0;
    int end = 0;
    int totalKmers = 0;
    int observedKmers = 0;
    int variations = 0;
    int kmerDistance = 0;

    void addVariationOriginal(int gapSize, int kmerSize)
    {
        variations += 1;
        int d = gapSize - (kmerSize - 1);
        if (d <= 0)
            d = std::abs(d + 1);
        kmerDistance += d;
    }
};
