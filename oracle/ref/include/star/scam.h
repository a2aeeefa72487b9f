/* Shim of star-camera 0.2 (TEST INFRASTRUCTURE ONLY): the camera ray of a
 * film/lens sample (pinhole, thin lens or orthographic). */
#ifndef REF_SHIM_SCAM_H
#define REF_SHIM_SCAM_H
#include <rsys/rsys.h>

struct scam;
struct scam_sample { double film[2]; double lens[2]; };
#define SCAM_SAMPLE_NULL__ {{0, 0}, {0, 0}}
static const struct scam_sample SCAM_SAMPLE_NULL = SCAM_SAMPLE_NULL__;
struct scam_ray { double org[3]; double dir[3]; };
#define SCAM_RAY_NULL__ {{0, 0, 0}, {0, 0, 0}}
static const struct scam_ray SCAM_RAY_NULL = SCAM_RAY_NULL__;

res_T scam_generate_ray(const struct scam* cam, const struct scam_sample* sample,
                        struct scam_ray* ray);
#endif
