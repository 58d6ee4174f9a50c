// host_order.hpp -- pattern-level set-up on the host: ABMC schedule, level
// schedules, permuted / lower-triangular patterns with value maps. These run
// once per sparsity pattern (cached by the solver objects); all value work
// (gathers, factorisation, solves) happens on the device.
#pragma once

#include <cstdint>
#include <vector>

namespace ssv {

// ABMCSchedule (include/sparsesolv/core/abmc_ordering.hpp:45-411): colours ->
// blocks -> rows, with rows of a block contiguous in the new numbering and
// colour c owning blocks color_offsets[c] .. color_offsets[c+1]-1.
struct AbmcSchedule {
    int num_colors = 0;
    int num_blocks = 0;
    std::vector<int> color_offsets;  // num_colors + 1
    std::vector<int> block_offsets;  // num_blocks + 1 (row ranges, new numbering)
    std::vector<int> ordering;       // ordering[old] = new
    std::vector<int> reverse;        // reverse[new] = old
};

void build_abmc(int n, const int* rp, const int* ci, int block_size, int target_colors,
                AbmcSchedule& out);

// Reverse Cuthill-McKee ordering (include/sparsesolv/core/rcm_ordering.hpp:
// 38-140): start at the first row of least degree, move twice to the first
// row at the largest BFS distance, then BFS from there with the unvisited
// neighbours of each row sorted by degree, unreached rows seeding further
// searches in index order, and reverse. ordering[old] = new, reverse[new] = old.
void rcm_order(int n, const int* rp, const int* ci, std::vector<int>& ordering, std::vector<int>& reverse);

// Level of every row for a forward (lower) or backward (upper) sweep
// (include/sparsesolv/core/level_schedule.hpp:58-135). Returns #levels.
int build_levels(int n, const int* rp, const int* ci, bool upper, std::vector<int>& level_of);

// Rows grouped by level: rows sorted by (level, index); offsets per level.
void group_by_level(const std::vector<int>& level_of, int nlev, std::vector<int>& rows,
                    std::vector<int>& offsets);

// Pattern of P A P^T (entry (i,j) -> (perm[i], perm[j]), rows sorted) and the
// source position of every new entry (ic_preconditioner.hpp:925-989).
void permute_pattern(int n, const int* rp, const int* ci, const int* perm, std::vector<int>& prp,
                     std::vector<int>& pci, std::vector<int>& src);

// Lower triangle incl. diagonal (ic_preconditioner.hpp:1075-1115) with source
// positions; U = L^T with, for every entry, its position in L
// (sparse_matrix_csr.hpp:47-72: rows of L^T list L rows in ascending order, so
// the diagonal comes first).
void lower_pattern(int n, const int* rp, const int* ci, std::vector<int>& lrp, std::vector<int>& lci,
                   std::vector<int>& lsrc);
void transpose_pattern(int n, const std::vector<int>& lrp, const std::vector<int>& lci,
                       std::vector<int>& urp, std::vector<int>& uci, std::vector<int>& usrc);

}  // namespace ssv
