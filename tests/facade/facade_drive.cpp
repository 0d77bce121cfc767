// Drives the reference-style C++ interface (include/smccat_particle.hpp) the
// way the reference's SMC driver does (src/main.cpp:55-106, 295-312): builds
// particles with the reference's constructor, runs Mcmc with the reference's
// move registry on each, then loads the final states into a shared batch with
// copyFromSerialized and runs the batched sweep. Every state and its
// log-likelihood / log-prior go to stdout as one JSON line, for the test to
// check against the CPU oracle.
//
// usage: facade_drive <input> <particles> <iterations> <temperature>
// input: int32 T, S, R, lg, invar, cat, then T*S residue codes (uint8).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <vector>

#include "smccat_particle.hpp"

namespace {

template <class V>
std::string json_list(const V& v) {
    std::ostringstream o;
    o.precision(17);
    o << "[";
    for (size_t i = 0; i < v.size(); ++i) o << (i ? "," : "") << v[i];
    o << "]";
    return o.str();
}

void emit(const char* phase, int index, smccat::Particle& p) {
    smccat::SerializedParticle sp;
    p.writeToSerialized(sp);
    std::vector<double> logits;
    for (const auto& l : sp.stationaries) logits.insert(logits.end(), l.begin(), l.end());
    std::ostringstream o;
    o.precision(17);
    o << "{\"phase\":\"" << phase << "\",\"index\":" << index << ",\"lnl\":" << p.lnLikelihood()
      << ",\"ln_prior\":" << p.lnPrior() << ",\"parent\":" << json_list(sp.parent)
      << ",\"branch\":" << json_list(sp.branchLengths) << ",\"base\":" << json_list(sp.baseMatrix)
      << ",\"num_classes\":" << sp.stationaries.size() << ",\"logits\":" << json_list(logits)
      << ",\"assign\":" << json_list(sp.assignments) << ",\"category_size\":" << json_list(sp.categorySize)
      << ",\"pinv\":" << sp.pInvar << ",\"shape\":" << sp.shape
      << ",\"move_count\":" << json_list(p.moveCount) << ",\"accept_count\":" << json_list(p.acceptCount)
      << ",\"splits\":" << p.getSplitSet().size() << "}";
    std::cout << o.str() << std::endl;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 5) {
        std::cerr << "usage: facade_drive <input> <particles> <iterations> <temperature>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t hdr[6];
    in.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
    const int T = hdr[0], S = hdr[1], R = hdr[2];
    const bool lg = hdr[3], invar = hdr[4], cat = hdr[5];
    std::vector<uint8_t> codes((size_t)T * S);
    in.read(reinterpret_cast<char*>(codes.data()), (std::streamsize)codes.size());
    if (!in) {
        std::cerr << "short input\n";
        return 2;
    }
    const int n = std::atoi(argv[2]), iterations = std::atoi(argv[3]);
    const double temperature = std::atof(argv[4]);
    try {
        std::vector<std::string> names;
        for (int t = 0; t < T; ++t) names.push_back("taxon" + std::to_string(t));
        smccat::Alignment aln(names, codes, S);
        smccat::SplitPosteriors splits;  // empty: every adaptive-NNI weight is epsilon + 1
        smccat::Mcmc mcmc;
        smccat::standardMoves(mcmc, aln, R, invar, lg, splits);

        // One Particle per "thread", the reference's constructor (main.cpp:112-115).
        std::vector<smccat::SerializedParticle> states(n);
        for (int i = 0; i < n; ++i) {
            smccat::Particle p(i + 1, aln, R, invar, lg, cat);
            emit("init", i, p);
            mcmc(p, iterations, temperature);
            emit("mcmc", i, p);
            if (cat) {
                p.gibbsPartitionMove(temperature);
                emit("gibbs", i, p);
            }
            p.writeToSerialized(states[i]);
        }

        // The same states in one shared batch, the batched sweep.
        smccat::ParticleBatch batch(aln, n, R, invar, lg, cat);
        std::vector<smccat::Particle> views;
        for (int i = 0; i < n; ++i) {
            views.emplace_back(100 + i, batch, i);
            views.back().copyFromSerialized(states[i]);
            emit("loaded", i, views.back());
        }
        mcmc(batch, iterations, temperature, 12345);
        for (int i = 0; i < n; ++i) emit("batch", i, views[i]);
    } catch (const smccat::Error& e) {
        std::cerr << e.what() << std::endl;
        return 3;
    }
    return 0;
}
