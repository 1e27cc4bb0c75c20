// Binomial checkpointing schedule (Griewank & Walther, "Algorithm 799: revolve",
// ACM TOMS 26(1), 2000).  The reference embeds the same published algorithm in
// Revolve<T>::revolve (lib/revolve.cpp:150-305); the schedule must match it
// action for action, so the decision rules below follow the published ones:
//   - a new checkpoint is taken whenever the current state is not yet stored;
//   - otherwise the next advance length is chosen from binomial coefficients
//     beta(ds, reps) of the remaining free snapshots ds and repetitions reps;
//   - the first reversal returns FIRSTURN, later ones YOUTURN;
//   - after a reversal the previous checkpoint is restored (RESTORE) until the
//     first one has been consumed (TERMINATE).
#include <climits>
#include "rsgpu.h"
#include "rsgpu_host.h"

namespace rsgpu {

static const int kCheckUp = 512;   // capacity of the checkpoint index table
static const int kRepsUp = 64;     // largest admissible repetition number

int RevolveSchedule::maxrange(int ss, int tt)
{
    // (ss+tt)! / (ss! tt!) evaluated in double, saturated at INT_MAX
    if (tt < 0 || ss < 0) return -1;
    double res = 1.0;
    for (int i = 1; i <= tt; i++) {
        res *= (ss + i);
        res /= i;
        if (res > INT_MAX) return INT_MAX;
    }
    return (int)res;
}

int RevolveSchedule::adjust(int steps)
{
    int snaps = 1, reps = 1, s = 0;
    while (maxrange(snaps + s, reps + s) > steps) s--;
    while (maxrange(snaps + s, reps + s) < steps) s++;
    snaps += s;
    reps += s;
    s = -1;
    while (maxrange(snaps, reps) >= steps) {
        if (snaps > reps) { snaps -= 1; s = 0; }
        else { reps -= 1; s = 1; }
    }
    if (s == 0) snaps += 1;
    if (s == 1) reps += 1;
    return snaps;
}

int RevolveSchedule::numforw(int steps, int snaps)
{
    if (snaps < 1 || snaps > kCheckUp) return -1;
    int reps = 0, range = 1;
    while (range < steps) {
        reps += 1;
        range = range * (reps + snaps) / reps;
    }
    if (reps > kRepsUp) return -1;
    return reps * steps - range * reps / (snaps + 1);
}

RevolveSchedule::RevolveSchedule(int steps, int snaps)
    : check_(-1), capo_(0), fine_(steps), steps_(steps), snaps_(snaps), info_(0), turn_(0), reps_(0), range_(0),
      oldsnaps_(0), oldfine_(0)
{
    // the reference falls back to adjust() for an invalid snapshot count (lib/revolve.cpp:12-15)
    if (snaps_ > steps_ || snaps_ < 2) snaps_ = adjust(steps_);
    for (int &c : ch_) c = 0;
}

int RevolveSchedule::next()
{
    if (check_ < -1 || capo_ > fine_) return RSGPU_ERROR;
    if (check_ == -1 && capo_ < fine_) {
        turn_ = 0;
        ch_[0] = capo_ - 1;
    }
    const int span = fine_ - capo_;
    if (span == 0) {
        // a reversal finished: fall back to the previous checkpoint, or stop
        if (check_ == -1 || capo_ == ch_[0]) {
            check_ -= 1;
            return RSGPU_TERMINATE;
        }
        capo_ = ch_[check_];
        oldfine_ = fine_;
        return RSGPU_RESTORE;
    }
    if (span == 1) {
        // one combined forward/adjoint step
        fine_ -= 1;
        if (check_ >= 0 && ch_[check_] == capo_) check_ -= 1;
        oldfine_ = fine_;
        if (turn_ == 0) {
            turn_ = 1;
            return RSGPU_FIRSTURN;
        }
        return RSGPU_YOUTURN;
    }
    if (check_ == -1 || ch_[check_] != capo_) {
        // the current state is not stored yet
        check_ += 1;
        if (check_ >= kCheckUp) { info_ = 10; return RSGPU_ERROR; }
        if (check_ + 1 > snaps_) { info_ = 11; return RSGPU_ERROR; }
        ch_[check_] = capo_;
        if (check_ == 0) {
            oldsnaps_ = snaps_;
            if (snaps_ > kCheckUp) { info_ = 14; return RSGPU_ERROR; }
        }
        oldfine_ = fine_;
        return RSGPU_TAKESHOT;
    }
    // advance: choose the next checkpoint position from the binomial table
    if (oldfine_ < fine_ && snaps_ == check_ + 1) { info_ = 13; return RSGPU_ERROR; }
    const int oldcapo = capo_;
    const int ds = snaps_ - check_;
    if (ds < 1) { info_ = 11; return RSGPU_ERROR; }
    reps_ = 0;
    range_ = 1;
    while (range_ < fine_ - capo_) {
        reps_ += 1;
        range_ = range_ * (reps_ + ds) / reps_;
    }
    if (reps_ > kRepsUp) { info_ = 15; return RSGPU_ERROR; }
    if (snaps_ != oldsnaps_ && snaps_ > kCheckUp) { info_ = 14; return RSGPU_ERROR; }
    const int bino1 = range_ * reps_ / (ds + reps_);
    const int bino2 = (ds > 1) ? bino1 * ds / (ds + reps_ - 1) : 1;
    int bino3;
    if (ds == 1) bino3 = 0;
    else bino3 = (ds > 2) ? bino2 * (ds - 1) / (ds + reps_ - 2) : 1;
    const int bino4 = bino2 * (reps_ - 1) / ds;
    int bino5;
    if (ds < 3) bino5 = 0;
    else bino5 = (ds > 3) ? bino3 * (ds - 2) / reps_ : 1;
    if (fine_ - capo_ <= bino1 + bino3) capo_ = capo_ + bino4;
    else if (fine_ - capo_ >= range_ - bino5) capo_ = capo_ + bino1;
    else capo_ = fine_ - bino2 - bino3;
    if (capo_ == oldcapo) capo_ = oldcapo + 1;
    oldfine_ = fine_;
    return RSGPU_ADVANCE;
}

}  // namespace rsgpu
