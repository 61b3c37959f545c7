"""The scene of the z-slab check: cube3d at 16^3 cells whose particles move
0.3 cells per step along z on top of the scene's random velocities, so that
particles cross the slab faces within a few steps (optionally with slip walls
on every face)."""


def scene(tb, walls: bool):
    sc = tb.scenes.cube3d(scale=16)
    dt, h = sc.params.dt, sc.mesh.h
    sc.particles.v[2] += 0.3 * h / dt
    if walls:
        sc.params.wall_mask = 0b111111
        sc.params.wall_layers = 2
    return sc
