// valmari_driver.cc -- builds Valmari's exact Markov-lumping minimiser
// (src/part_ref/MDP_minimize.cc with its reader MDP_read.cc), UNMODIFIED,
// into a binary that also prints the final block of every state.
//
// TEST INFRASTRUCTURE ONLY (it is the checker, never the product).
//
// The reference sources are #included from the reference tree at compile time
// (oracle/Makefile passes -I<reference>/src/part_ref); none is copied here.
// The glue below plays the part of src/part_ref/MDPmin.cc:105-170 (integer
// weights, or double weights when built with -DORC_F64; the store_* name
// mapping): it has to present the same interface to MDP_read.cc, and is
// written here in its minimal form.
//
// Input (stdin): the MDP text of MDP_read.cc:51-63, i.e.
//   "nr_states 0 0 nr_w_trans nr_blocks", then nr_w_trans lines "tail w head"
//   (1-based), then for blocks 2..nr_blocks the member states followed by 0.
// Output (stdout): the minimiser's own three lines (MDP_minimize.cc:814-816),
//   then "labels b1 b2 ... bn" with b = which_block(state) for states 1..n.
#include <climits>
#include <iostream>
#include <sstream>
#include <string>

#ifdef ORC_F64
// the minimiser's double-weight configuration (MDPmin.cc:107-113): weights
// read as decimals, block sums rounded to float before they are compared
#include <cfloat>
#define MDP_weight_is_double
typedef double MDP_weight_type;
const MDP_weight_type MDP_zero_weight = 0.0, MDP_unused_weight = DBL_MAX;
inline void MDP_round_weight(MDP_weight_type& ww) { ww = float(ww); }
#else
typedef int MDP_weight_type;
const MDP_weight_type MDP_zero_weight = 0, MDP_unused_weight = INT_MIN;
inline void MDP_round_weight(MDP_weight_type&) {}
#endif

#include "MDP_minimize.cc"

inline void MDP_store_sizes(unsigned s, unsigned l, unsigned lt, unsigned wt, unsigned b)
{ MDPmin::store_sizes(s, l, lt, wt, b); }
inline void MDP_store_l_transition(unsigned t, unsigned l, unsigned h)
{ MDPmin::store_l_transition(t, l, h); }
inline void MDP_store_w_transition(unsigned t, const MDP_weight_type& w, unsigned h)
{ MDPmin::store_w_transition(t, w, h); }
inline void MDP_store_block(unsigned s, unsigned b) { MDPmin::store_block(s, b); }

#include "MDP_read.cc"

int main()
{
    std::ios::sync_with_stdio(false);
    std::string text((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
    unsigned n = 0;
    { std::istringstream head(text); head >> n; }
    std::istringstream body(text);
    reader input(&body);
    MDP_read(input);
    MDPmin::minimize();
    std::fflush(stdout);
    std::string line = "labels";
    for (unsigned s = 1; s <= n; ++s) { line += ' '; line += std::to_string(MDPmin::which_block(s)); }
    line += '\n';
    std::fputs(line.c_str(), stdout);
    MDPmin::terminate();
    return 0;
}
