// qreducer.h -- streaming forall/exists reducer over items pushed in index
// order (the semantics of QuantReducer, qsat.rs:172-291), used by the host to
// combine per-launch results over the quantifiers above one launch.
#pragma once
#include <cstdint>
#include <vector>

namespace nsat {

struct FinalResult {
    bool reversed = false;      // first quantifier is All
    uint32_t solution_bits = 0;
    bool has_solution = false;
    uint64_t solution = 0;      // bit k = input k of the first block
};

class QuantReducer {
public:
    // quants[i] for inputs 0..nq-1 (1 = All); nq in 1..64
    explicit QuantReducer(const std::vector<uint8_t>& quants) {
        nq_ = (int)quants.size();
        int fb = 0;
        while (fb < nq_ && quants[fb] == quants[0]) fb++;
        first_bits_ = fb;
        q_.resize(nq_);
        r_.resize(nq_);
        for (int i = 0; i < nq_; i++) { q_[i] = quants[nq_ - 1 - i]; r_[i] = q_[i]; }
        all_mask_ = nq_ == 64 ? ~0ull : ((1ull << nq_) - 1);
        const uint64_t fm = fb >= 64 ? ~0ull : ((1ull << fb) - 1);
        first_mask_ = (nq_ - fb) >= 64 ? 0 : (fm << (nq_ - fb));
        other_mask_ = all_mask_ & ~first_mask_;
    }

    bool is_end() const { return started_ && (start_ & all_mask_) == 0; }
    uint64_t next_index() const { return start_; }

    // Pushes the item with index next_index().
    void push(bool item) {
        started_ = true;
        uint64_t index = start_;
        uint8_t prev = item ? 1 : 0;
        for (int i = 0; i < nq_; i++) {
            const uint8_t q = q_[i], r = r_[i];
            prev = (uint8_t)((r & prev) | ((r ^ prev) & (q ^ 1)));
            r_[i] = prev;
            if ((index & 1) == 0) break;
            index >>= 1;
            r_[i] = q;
        }
        if (!has_solution_ && (start_ & other_mask_) == other_mask_ && (prev ^ q_[nq_ - 1])) {
            const uint64_t v = start_ >> (nq_ - first_bits_);
            uint64_t rev = 0;
            for (int k = 0; k < first_bits_; k++) rev |= ((v >> k) & 1ull) << (first_bits_ - 1 - k);
            has_solution_ = true;
            solution_ = rev;
        }
        start_ += 1;
    }

    bool final_result(FinalResult* out) const {
        if (!(is_end() || has_solution_)) return false;
        out->reversed = q_[nq_ - 1] != 0;
        out->solution_bits = (uint32_t)first_bits_;
        out->has_solution = has_solution_;
        out->solution = has_solution_ ? solution_ : 0;
        return true;
    }

private:
    int nq_ = 0, first_bits_ = 0;
    std::vector<uint8_t> q_, r_;
    bool started_ = false, has_solution_ = false;
    uint64_t start_ = 0, all_mask_ = 0, first_mask_ = 0, other_mask_ = 0, solution_ = 0;
};

}  // namespace nsat
