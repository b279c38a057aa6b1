/* hm_tune.h - the launch-shape table filled by hm_autotune */
#ifndef HM_TUNE_H
#define HM_TUNE_H

namespace hm
{
struct TuneEntry
{
  int   tpb, radius, rows; /* vpipes: fused-kernel launch shape; thermal: rows per CTA */
  int   block;             /* thermal: steps per launch                                */
  float ms_per_step;
};
/* the tuned shape for this grid's size class, if any */
bool tuned_vpipes(int nx, int ny, TuneEntry *out);
bool tuned_thermal(int nx, int ny, TuneEntry *out);
/* the batched form's tuned choice (tpb: persistent CTAs per SM, rows:
 * thermal tile rows), if any */
bool tuned_batch(TuneEntry *out);
} // namespace hm

#endif
