/* orc_types.h -- TEST INFRASTRUCTURE ONLY: types shared by the CPU oracle's sources. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pixel model of a sensor (Sensor.h:213-250): frustum constants or laser tables. */
typedef struct {
  int32_t type;  /* 0 frustum, 1 laser */
  int32_t width, height, pad;
  float hw, hh, c0, c1, scale_u, scale_v;
  float min_range, max_range;
  const float* sinu;
  const float* cosu;
  const float* sinv;
  const float* cosv;
} orc_sensor;

#ifdef __cplusplus
}
#endif
