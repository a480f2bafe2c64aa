"""The sun and the day/night cycle of cube-tracing's host (src/main.cpp),
for callers that drive the frame's point light and sky the way the
reference application does.

The frame kernels only read the results: LIGHT.position / LIGHT.emissive of
point light 0 and Status.time / Status.is_afternoon, which select the sky
colour (mat.glsl:137-202).  Arithmetic is single precision, as in the
reference's C++ (glm::mix(x, y, a) = x * (1 - a) + y * a).
"""
import numpy as np

from . import layouts as L

SUN_MAX_INTENSITY = np.float32(10000.0)                          # shared.inl:33
SUN_TOP_POSITION = np.array([0.0, 15.0, -5.0], np.float32)       # shared.inl:34-36
SUNSET_POSITION = np.array([20.0, 0.0, 0.0], np.float32)         # main.cpp:184
DAY_DURATION = np.float32(60.0)                                  # main.cpp:37, seconds


def _mix(x, y, a):
    a = np.float32(a)
    return (x * (np.float32(1.0) - a) + y * a).astype(np.float32)


def sun_position(t, is_afternoon):
    """interpolate_sun_light (main.cpp:180-213): from the sunset (afternoon)
    or its mirror (morning) at t = 0 to the top position at t = 1."""
    start = SUNSET_POSITION if is_afternoon else -SUNSET_POSITION
    return _mix(start, SUN_TOP_POSITION, t)


def sun_intensity(t, is_afternoon, max_intensity=SUN_MAX_INTENSITY, min_intensity=0.0):
    """interpolate_sun_intensity (main.cpp:215-232): dark before t = 0.5,
    then mix(0, max, t)."""
    t = np.float32(t)
    if t >= np.float32(0.5):
        return np.float32(np.float32(0.0) * (np.float32(1.0) - t) + np.float32(max_intensity) * t)
    return np.float32(0.0)


def add_time(time, is_afternoon, dt):
    """add_time (main.cpp:440-444): time runs forward in the afternoon and
    backward in the morning."""
    return np.float32(np.float32(time) + np.float32(dt) * np.float32(1.0 if is_afternoon else -1.0))


def update_sun(time, is_afternoon, point_lights):
    """update_sun_light (main.cpp:497-510): past either end of [0, 1] the
    half of the day flips and the time is clamped; point light 0 becomes the
    sun.  Returns the new (time, is_afternoon); `point_lights` (a LIGHT array)
    is updated in place."""
    time = np.float32(time)
    if time < 0.0 or time > 1.0:
        is_afternoon = not is_afternoon
        time = np.float32(min(max(float(time), 0.0), 1.0))
    point_lights[0]["position"] = sun_position(time, is_afternoon)
    i = sun_intensity(time, is_afternoon)
    point_lights[0]["emissive"] = (i, i, i)
    return time, is_afternoon


def make_sun(point_lights_count=1):
    """create_point_lights (main.cpp:349-379): one point light at the top
    position, full intensity, at midday (time 1, afternoon)."""
    pl = np.zeros(point_lights_count, L.LIGHT)
    pl["position"] = SUN_TOP_POSITION
    pl["emissive"] = (SUN_MAX_INTENSITY,) * 3
    pl["instance_id"] = L.MAX_INSTANCES
    pl["primitive_id"] = L.MAX_PRIMITIVES
    pl["type"] = L.LIGHT_POINT
    return pl, np.float32(1.0), True
