"""Procedural scenes in the reference's vision_scene.json schema.

box_room(): the plain-tracer workload — a unit box room of 10 triangles
(floor, ceiling, back, left, right walls as quads), a 0.3 x 0.6 x 0.3 box
rotated +15 degrees and a 0.3 x 0.3 x 0.3 box rotated -18 degrees about y
(12 triangles each, the `cube` shape), a 0.25 x 0.25 ceiling quad light, a
pinhole camera with fov_y 40, 256 x 256, 16 spp, max depth 8 and 4 hero
wavelengths.  The light is a 6500 K blackbody scaled to radiance 17, or its
RGB twin [17, 17, 17] (the reference's own illumination slot) when
rgb_light=True.
"""
import math

LEFT_RGB = [0.63, 0.065, 0.05]
RIGHT_RGB = [0.14, 0.45, 0.091]
GREY_RGB = [0.725, 0.725, 0.725]


def _cols(c0, c1, c2, t):
    """matrix4x4 in the schema's column order (fourth column = translation)."""
    return {"type": "matrix4x4", "param": {"matrix4x4": [list(c0) + [0.0], list(c1) + [0.0], list(c2) + [0.0],
                                                         list(t) + [1.0]]}}


def _ry(deg, t):
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    return _cols((c, 0.0, -s), (0.0, 1.0, 0.0), (s, 0.0, c), t)


def box_room(width=256, height=256, max_depth=8, min_depth=5, rr_threshold=1.0, dimension=4,
             sampler="independent", seed=0, rgb_light=False, light_scale=17.0):
    quad = lambda name, mat, xf, w=1.0, h=1.0: {"type": "quad", "name": name,
                                                 "param": {"width": w, "height": h, "material": mat, "transform": xf}}
    shapes = [
        quad("floor", "Floor", _cols((1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, 0))),
        quad("ceiling", "Ceiling", _cols((1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 1, 0))),
        quad("back", "BackWall", _cols((1, 0, 0), (0, 0, 1), (0, -1, 0), (0, 0.5, -0.5))),
        quad("left", "LeftWall", _cols((0, -1, 0), (1, 0, 0), (0, 0, 1), (-0.5, 0.5, 0))),
        quad("right", "RightWall", _cols((0, 1, 0), (-1, 0, 0), (0, 0, 1), (0.5, 0.5, 0))),
        {"type": "cube", "name": "tall_box",
         "param": {"x": 0.3, "y": 0.6, "z": 0.3, "material": "TallBox", "transform": _ry(15.0, (-0.17, 0.3, -0.13))}},
        {"type": "cube", "name": "short_box",
         "param": {"x": 0.3, "y": 0.3, "z": 0.3, "material": "ShortBox", "transform": _ry(-18.0, (0.17, 0.15, 0.12))}},
    ]
    if rgb_light:
        color = {"channels": "xyz", "node": [light_scale] * 3}
        scale = 1.0
    else:
        color = {"channels": "xyz", "node": {"type": "blackbody", "param": {"temperature": 6500.0}}}
        scale = light_scale
    shapes.append({"type": "quad", "name": "light",
                   "param": {"width": 0.25, "height": 0.25, "material": "Light",
                             "transform": _cols((1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0.999, 0)),
                             "emission": {"type": "area", "param": {"color": color, "scale": scale,
                                                                    "two_sided": False}}}})
    materials = [
        {"type": "diffuse", "name": "Floor", "param": {"color": GREY_RGB}},
        {"type": "diffuse", "name": "Ceiling", "param": {"color": GREY_RGB}},
        {"type": "diffuse", "name": "BackWall", "param": {"color": GREY_RGB}},
        {"type": "diffuse", "name": "LeftWall", "param": {"color": LEFT_RGB}},
        {"type": "diffuse", "name": "RightWall", "param": {"color": RIGHT_RGB}},
        {"type": "diffuse", "name": "TallBox", "param": {"color": GREY_RGB}},
        {"type": "diffuse", "name": "ShortBox", "param": {"color": GREY_RGB}},
        {"type": "black_body", "name": "Light", "param": {}},
    ]
    return {
        "shapes": shapes,
        "materials": materials,
        "camera": {"type": "pinhole", "param": {
            "fov_y": 40.0,
            "transform": {"type": "look_at", "param": {"position": [0.0, 0.5, 1.85], "target_pos": [0.0, 0.5, 0.0],
                                                       "up": [0.0, 1.0, 0.0]}},
            "radiance_collector": {"type": "normal", "param": {"resolution": [width, height], "exposure": 1.0}},
            "filter": {"type": "box", "param": {"radius": [0.5, 0.5]}}}},
        "integrator": {"type": "pt", "param": {"max_depth": max_depth, "min_depth": min_depth,
                                               "rr_threshold": rr_threshold}},
        "spectrum": {"type": "hero", "param": {"dimension": dimension}},
        "sampler": {"type": sampler, "param": {"seed": seed}},
        "light_sampler": {"type": "uniform", "param": {"lights": []}},
        "render_setting": {"polymorphic_mode": 1},
    }


def material_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with the microfacet materials on its objects: a gold
    conductor tall box, a dispersive glass short box (Cauchy A = 1.5,
    B = 0.0042) and a principled floor."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    mats["TallBox"].update({"type": "metal", "param": {"material_name": "Au", "roughness": 0.3}})
    mats["ShortBox"].update({"type": "glass", "param": {
        "color": [1.0, 1.0, 1.0], "roughness": 0.2,
        "ior": {"type": "cauchy", "param": {"A": 1.5, "B": 0.0042}}}})
    mats["Floor"].update({"type": "principled_bsdf", "param": {
        "color": [0.8, 0.5, 0.3], "metallic": 0.4, "roughness": 0.35}})
    return sc


def substrate_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with the remaining reference materials: a near-specular
    tinted mirror tall box, a glossy substrate short box (roughness remapped)
    and a substrate floor with plain alphas (the reference's coffee-scene
    plastics: Rd, Rs 0.05 default, roughness 0.1 unremapped)."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    mats["TallBox"].update({"type": "mirror", "param": {"color": [0.95, 0.9, 0.8], "roughness": 0.05}})
    mats["ShortBox"].update({"type": "substrate", "param": {
        "color": [0.2, 0.4, 0.8], "spec": [0.08, 0.08, 0.08], "roughness": 0.6}})
    mats["Floor"].update({"type": "substrate", "param": {
        "color": [0.58, 0.58, 0.58], "roughness": [0.1, 0.1], "remapping_roughness": False}})
    return sc


def metallic_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with `metallic` materials (MetallicMaterial: colour as F0
    and reflectance, F82 edge tint): a warm tall box, an anisotropic short
    box with a blue edge tint and a near-specular back wall."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    mats["TallBox"].update({"type": "metallic", "param": {"color": [0.95, 0.64, 0.37], "edge_tint": [1.0, 0.85, 0.7],
                                                          "roughness": 0.35}})
    mats["ShortBox"].update({"type": "metallic", "param": {"color": [0.8, 0.82, 0.85], "edge_tint": [0.6, 0.7, 1.0],
                                                           "roughness": 0.3, "anisotropic": 0.5}})
    mats["BackWall"].update({"type": "metallic", "param": {"color": [0.9, 0.9, 0.9], "roughness": 0.1}})
    return sc


def principled_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with principled BSDFs that use every layer: a sheen-and-
    coat tall box over a metallic base, a transmissive short box with a coat,
    and a sheen floor (PrincipledBSDF's sheen LTC, coat, metallic,
    transmission, specular and diffuse lobes)."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    mats["TallBox"].update({"type": "principled_bsdf", "param": {
        "color": [0.7, 0.3, 0.2], "metallic": 0.5, "roughness": 0.4, "spec_tint": [0.9, 0.9, 1.0],
        "sheen_weight": 0.8, "sheen_roughness": 0.4, "sheen_tint": [0.9, 0.8, 0.6],
        "coat_weight": 0.7, "coat_roughness": 0.15, "coat_ior": 1.6, "coat_tint": [0.95, 0.95, 0.9]}})
    mats["ShortBox"].update({"type": "principled_bsdf", "param": {
        "color": [0.85, 0.9, 0.95], "roughness": 0.25, "ior": 1.45, "transmission_weight": 0.8,
        "coat_weight": 0.3, "coat_roughness": 0.1}})
    mats["Floor"].update({"type": "principled_bsdf", "param": {
        "color": [0.5, 0.45, 0.4], "roughness": 0.6, "sheen_weight": 1.0, "sheen_roughness": 0.7,
        "sheen_tint": [0.6, 0.7, 0.9]}})
    return sc


def plastic_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with plastic boxes (PlasticLobe): a glossy blue short box
    (ior 1.5, roughness 0.3) and a near-specular white tall box (roughness
    0.1, remapped twice to alpha 1e-4)."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    mats["ShortBox"].update({"type": "plastic", "param": {
        "color": [0.1, 0.2, 0.7], "spec": [1.0, 1.0, 1.0], "ior": 1.5, "roughness": 0.3}})
    mats["TallBox"].update({"type": "plastic", "param": {"color": [0.8, 0.8, 0.8], "roughness": 0.1}})
    return sc


def mix_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8):
    """The box room with mix and add materials (MixMaterial / AddMaterial):
    the tall box mixes two BK7 glasses half and half (the reference's
    cbox/vision_scene.json `mix` material), the short box mixes a diffuse
    and a gold conductor (frac 0.3), the floor adds a diffuse and a coated
    principled BSDF, the back wall mixes a plastic and a substrate (frac
    0.6)."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    glass = {"type": "glass", "param": {"material_name": "BK7", "color": {"channels": "xyz", "node": [1, 1, 1]},
                                        "roughness": [0.001, 0.001]}}
    mats["TallBox"].update({"type": "mix", "param": {"mat0": glass, "mat1": dict(glass)}})
    mats["ShortBox"].update({"type": "mix", "param": {
        "frac": 0.3,
        "mat0": {"type": "diffuse", "param": {"color": [0.7, 0.3, 0.2]}},
        "mat1": {"type": "metal", "param": {"material_name": "Au", "roughness": 0.2}}}})
    mats["Floor"].update({"type": "add", "param": {
        "mat0": {"type": "diffuse", "param": {"color": [0.3, 0.3, 0.35]}},
        "mat1": {"type": "principled_bsdf", "param": {"color": [0.6, 0.5, 0.4], "metallic": 0.2, "roughness": 0.4,
                                                      "coat_weight": 0.5, "coat_roughness": 0.1}}}})
    mats["BackWall"].update({"type": "mix", "param": {
        "frac": 0.6,
        "mat0": {"type": "plastic", "param": {"color": [0.2, 0.4, 0.7], "roughness": 0.2}},
        "mat1": {"type": "substrate", "param": {"color": [0.6, 0.5, 0.3], "roughness": 0.3}}}})
    return sc


ROOM_TEXTURES = ("checker.png", "gradient.png", "photo.jpg")


def textured_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8, jpeg=True):
    """The box room with `image` shader nodes in its colour slots: the back
    wall is a diffuse with an RGB image, the floor a diffuse whose colour is
    multiply(image, constant) with a grey image, the short box a principled
    BSDF with the JPEG image (jpeg=False: the RGB image) and the tall box a
    plastic with the grey image.  The files (ROOM_TEXTURES) are looked up in
    the scene's base folder."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    mats = {m["name"]: m for m in sc["materials"]}
    img = lambda fn, **kw: {"type": "image", "param": dict(fn=fn, **kw)}
    mats["BackWall"]["param"] = {"color": {"channels": "xyz", "node": img("checker.png")}}
    mats["Floor"]["param"] = {"color": {"channels": "xyz", "node": {"type": "multiply", "param": {
        "lhs": img("gradient.png"), "rhs": [0.8, 0.7, 0.6]}}}}
    mats["ShortBox"].update({"type": "principled_bsdf", "param": {
        "color": img("photo.jpg" if jpeg else "checker.png"), "metallic": 0.1, "roughness": 0.5}})
    mats["TallBox"].update({"type": "plastic", "param": {
        "color": img("gradient.png", color_space="linear"), "roughness": 0.2}})
    return sc


def projector_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8, light_sampler="uniform",
                   area_light=False):
    """The box room lit by two projectors (Projector): one casts the RGB
    image of textured_room's files (checker.png, its aspect ratio) onto the
    back wall, the other a constant warm colour onto the floor through a
    wide 1.5 : 1 frustum; with or without the room's area light."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    if not area_light:
        sc["shapes"] = [s for s in sc["shapes"] if s["name"] != "light"]
    look = lambda pos, target: {"type": "look_at", "param": {"position": pos, "target_pos": target, "up": [0, 1, 0]}}
    image = {"type": "projector", "param": {
        "color": {"channels": "xyz", "node": {"fn": "checker.png", "color_space": "srgb"}},
        "angle": 14.0, "ratio": 0, "scale": 3.0, "o2w": look([0.1, 0.55, 1.2], [0.0, 0.5, -0.5])}}
    warm = {"type": "projector", "param": {
        "color": {"channels": "xyz", "node": [1.0, 0.7, 0.4]}, "angle": 25.0, "ratio": 1.5, "scale": 0.6,
        "o2w": look([0.0, 0.95, 0.3], [0.05, 0.0, 0.1])}}
    sc["light_sampler"] = {"type": light_sampler, "param": {"lights": [image, warm]}}
    return sc


def point_light_room(width=64, height=64, dimension=4, sampler="independent", max_depth=8, light_sampler="uniform",
                     area_light=True):
    """The box room lit by a white point light near the ceiling and a warm
    spot light aimed at the short box (PointLight / SpotLight of the light
    sampler's list), with or without the room's area light."""
    sc = box_room(width=width, height=height, dimension=dimension, sampler=sampler, max_depth=max_depth)
    if not area_light:
        sc["shapes"] = [s for s in sc["shapes"] if s["name"] != "light"]
    point = {"type": "point", "param": {"color": {"channels": "xyz", "node": [1.0, 1.0, 1.0]},
                                        "position": [-0.2, 0.9, 0.1], "scale": 0.15}}
    spot = {"type": "spot", "param": {"color": {"channels": "xyz", "node": [1.0, 0.8, 0.5]},
                                      "position": [0.35, 0.95, 0.4], "direction": [-0.3, -1.0, -0.4],
                                      "angle": 30.0, "falloff": 12.0, "scale": 0.4}}
    sc["light_sampler"] = {"type": light_sampler, "param": {"lights": [point, spot]}}
    return sc


def _draw_material(rng, name):
    """One of the three material families, drawn uniformly, with the
    parameter distributions of the large-scene workload."""
    kind = rng.integers(0, 3)
    if kind == 0:
        return {"type": "metal", "name": name,
                "param": {"material_name": "Au", "roughness": float(rng.uniform(0.05, 0.5))}}
    if kind == 1:
        return {"type": "glass", "name": name,
                "param": {"color": [1.0, 1.0, 1.0], "roughness": 0.01,
                          "ior": {"type": "cauchy", "param": {"A": 1.5, "B": 0.0042}}}}
    return {"type": "principled_bsdf", "name": name,
            "param": {"color": [float(x) for x in rng.uniform(0.0, 1.0, 3)],
                      "metallic": float(rng.uniform(0.0, 1.0)),
                      "roughness": float(rng.uniform(0.1, 0.9))}}


def large_scene(width=1024, height=1024, max_depth=16, dimension=4, sampler="pcg", seed=1,
                subdivisions=7, grid=1000, tiles=10, sky_width=2048, sky_height=1024):
    """Seeded large scene: a displaced subdivided icosphere (value-noise
    displacement of amplitude 0.05, seed 1) on a grid x grid ground split into
    tiles x tiles objects; per-object materials drawn uniformly from a GGX gold
    conductor (roughness U[0.05, 0.5]), a dispersive glass (Cauchy A = 1.5,
    B = 0.0042) and a principled BSDF (baseColor U[0,1]^3, metallic U[0,1],
    roughness U[0.1, 0.9]); lit by a procedural 2048 x 1024 HDR sky
    (gradient plus a 5-degree sun lobe peaking at 5e4)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    materials = [_draw_material(rng, "sphere_mat")]
    shapes = [{"type": "icosphere", "name": "sphere",
               "param": {"subdivisions": subdivisions, "radius": 1.0, "material": "sphere_mat",
                         "displacement": {"amplitude": 0.05, "frequency": 4.0, "seed": seed},
                         "transform": _cols((1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1.0, 0))}}]
    extent = 40.0
    per = grid // tiles
    tsize = extent / tiles
    for j in range(tiles):
        for i in range(tiles):
            name = "ground_%d_%d" % (i, j)
            materials.append(_draw_material(rng, name + "_mat"))
            cx = -extent / 2 + (i + 0.5) * tsize
            cz = -extent / 2 + (j + 0.5) * tsize
            shapes.append({"type": "grid", "name": name,
                           "param": {"nx": per, "nz": per, "size_x": tsize, "size_z": tsize,
                                     "material": name + "_mat",
                                     "transform": _cols((1, 0, 0), (0, 1, 0), (0, 0, 1), (cx, 0.0, cz))}})
    sky = {"type": "spherical", "param": {
        "color": {"channels": "xyz", "node": {"type": "sky", "param": {
            "width": sky_width, "height": sky_height, "sun_elevation": 35.0, "sun_azimuth": 40.0,
            "sun_radius": 5.0, "sun_peak": 5e4}}},
        "scale": 1.0}}
    return {
        "shapes": shapes,
        "materials": materials,
        "camera": {"type": "pinhole", "param": {
            "fov_y": 40.0,
            "transform": {"type": "look_at", "param": {"position": [0.0, 2.2, 5.0], "target_pos": [0.0, 0.9, 0.0],
                                                       "up": [0.0, 1.0, 0.0]}},
            "radiance_collector": {"type": "normal", "param": {"resolution": [width, height], "exposure": 1.0}},
            "filter": {"type": "box", "param": {"radius": [0.5, 0.5]}}}},
        "integrator": {"type": "pt", "param": {"max_depth": max_depth, "min_depth": 5, "rr_threshold": 1.0}},
        "spectrum": {"type": "hero", "param": {"dimension": dimension}},
        "sampler": {"type": sampler, "param": {"seed": 0}},
        "light_sampler": {"type": "uniform", "param": {"lights": [sky]}},
        "render_setting": {"polymorphic_mode": 1},
    }


def _rot_m(axis, deg):
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    import numpy as np
    m = np.eye(4)
    if axis == 'x':
        m[1, 1], m[1, 2], m[2, 1], m[2, 2] = c, -s, s, c
    else:
        m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    return m


def camera_c2w(position, target, up=(0.0, 1.0, 0.0)):
    """Camera-to-world matrix (row-major 4x4) that the scene loader builds from
    a look_at transform: the sensor keeps yaw and pitch of the look-at frame and
    composes T(position) * scale(1, 1, -1) * Ry(yaw) * Rx(-pitch)."""
    import numpy as np
    pos, tgt, up = (np.asarray(v, np.float64) for v in (position, target, up))
    fwd = tgt - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    up2 = np.cross(right, fwd)
    # look_at columns: right, up, forward; pitch/yaw as Sensor::update_mat reads them.
    pitch = math.degrees(math.atan2(up2[2], up2[1]))
    yaw = math.degrees(math.atan2(fwd[0], right[0]))
    t = np.eye(4)
    t[:3, 3] = pos
    sc = np.diag([1.0, 1.0, -1.0, 1.0])
    return (t @ sc @ _rot_m('y', yaw) @ _rot_m('x', -pitch)).astype(np.float32)


def camera_spline(frames=64, seed=3, target=(0.0, 0.45, 0.0)):
    """Seeded camera path for the many-light workload: a Catmull-Rom spline
    through 6 control points in front of the box room's open side
    (x in [-0.15, 0.15], y in [0.35, 0.65], z in [1.45, 1.95]), looking at the
    room centre.  Returns `frames` camera-to-world matrices."""
    import numpy as np
    rng = np.random.default_rng(seed)
    ctrl = np.stack([rng.uniform(-0.15, 0.15, 6), rng.uniform(0.35, 0.65, 6), rng.uniform(1.45, 1.95, 6)], 1)
    out = []
    for f in range(frames):
        t = f / max(frames - 1, 1) * (len(ctrl) - 3)
        i = min(int(t), len(ctrl) - 4)
        u = t - i
        p0, p1, p2, p3 = ctrl[i:i + 4]
        pos = 0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u +
                     (-p0 + 3 * p1 - 3 * p2 + p3) * u ** 3)
        out.append(camera_c2w(pos, target))
    return out


def many_lights(width=1920, height=1080, emitters=10000, seed=7, M_light=32, M_bsdf=1, history_limit=20,
                spatial_neighbours=5, spatial_radius=30.0, max_depth=8, sampler="pcg", gi=True, integrator="rt",
                dimension=3):
    """Many-light ReSTIR workload: the box room plus `emitters` one-sided
    emissive triangles (equilateral, edge U[0.01, 0.05], centres uniform in the
    room, random orientation, 2000-9000 K blackbody spectra, scale log-uniform
    over [1, 100]) with power-distribution light selection, rendered by the
    real-time ReSTIR integrator on 3 hero wavelengths: 32 initial light
    candidates, temporal reuse capped at M = 20, one spatial pass of 5
    neighbours within 30 pixels.  integrator="pt" keeps the plain path tracer
    (the geometry and emitters of the workload for other uses)."""
    import numpy as np
    sc = box_room(width=width, height=height, max_depth=max_depth, dimension=dimension, sampler=sampler, seed=0)
    rng = np.random.default_rng(seed)
    shapes = sc["shapes"]
    for i in range(emitters):
        edge = rng.uniform(0.01, 0.05)
        c = rng.uniform([-0.5, 0.0, -0.5], [0.5, 1.0, 0.5])
        # Random orthonormal frame: normal uniform on the sphere, in-plane angle uniform.
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        a = np.cross(n, [1.0, 0.0, 0.0] if abs(n[0]) < 0.9 else [0.0, 1.0, 0.0])
        a /= np.linalg.norm(a)
        b = np.cross(n, a)
        th = rng.uniform(0.0, 2.0 * math.pi)
        r = edge / math.sqrt(3.0)
        verts = [c + r * (math.cos(th + k * 2.0 * math.pi / 3.0) * a + math.sin(th + k * 2.0 * math.pi / 3.0) * b)
                 for k in range(3)]
        temp = float(rng.uniform(2000.0, 9000.0))
        scale = float(math.exp(rng.uniform(math.log(1.0), math.log(100.0))))
        shapes.append({"type": "mesh", "name": "emitter_%d" % i,
                       "param": {"positions": [float(x) for v in verts for x in v], "indices": [0, 1, 2],
                                 "material": "Light",
                                 "emission": {"type": "area", "param": {
                                     "color": {"channels": "xyz",
                                               "node": {"type": "blackbody", "param": {"temperature": temp}}},
                                     "scale": scale, "two_sided": False}}}})
    sc["light_sampler"] = {"type": "power", "param": {"lights": []}}
    if integrator == "pt":
        return sc
    sc["integrator"] = {"type": "rt", "param": {
        "max_depth": max_depth, "min_depth": 5, "rr_threshold": 1.0,
        "direct": {"M_light": M_light, "M_bsdf": M_bsdf,
                   "spatial": {"sample_num": spatial_neighbours, "radius": spatial_radius},
                   "temporal": {"history_limit": history_limit}},
        "indirect": {"open": bool(gi),
                     "spatial": {"sample_num": spatial_neighbours, "radius": spatial_radius},
                     "temporal": {"history_limit": history_limit}}}}
    return sc


def instanced_scene(width=1024, height=1024, copies=64, seed=11, subdivisions=6, patch=200, max_depth=16,
                    dimension=4, sampler="pcg"):
    """Serving scene of ~10 M triangles: `copies` instances of one mesh group
    modelled on the large scene's geometry (a displaced icosphere with
    `subdivisions` levels, 81,920 triangles at 6, on a `patch` x `patch` grid
    tile, 80,000 triangles at 200), each with a random position on an 8 x 8
    layout, y rotation and scale, and a material drawn like the large scene's;
    lit by the same procedural sky.  64 copies give 10,362,880 triangles of two
    distinct meshes, so the scene is traced through a two-level BVH (one BVH8
    per mesh under a top level over the 128 instances)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    shapes, materials = [], []
    side = int(math.ceil(math.sqrt(copies)))
    spacing = 4.0
    for c in range(copies):
        gx, gz = c % side, c // side
        cx = (gx - (side - 1) / 2.0) * spacing + rng.uniform(-0.5, 0.5)
        cz = (gz - (side - 1) / 2.0) * spacing + rng.uniform(-0.5, 0.5)
        s = float(rng.uniform(0.5, 1.5))
        ang = float(rng.uniform(0.0, 360.0))
        a = math.radians(ang)
        ca, sa = math.cos(a), math.sin(a)
        mat = _draw_material(rng, "copy_%d_mat" % c)
        materials.append(mat)
        rot = ((ca * s, 0.0, -sa * s), (0.0, s, 0.0), (sa * s, 0.0, ca * s))
        shapes.append({"type": "icosphere", "name": "copy_%d_sphere" % c,
                       "param": {"subdivisions": subdivisions, "radius": 1.0, "material": mat["name"],
                                 "displacement": {"amplitude": 0.05, "frequency": 4.0, "seed": seed},
                                 "transform": _cols(rot[0], rot[1], rot[2], (cx, s, cz))}})
        shapes.append({"type": "grid", "name": "copy_%d_ground" % c,
                       "param": {"nx": patch, "nz": patch, "size_x": spacing * 0.9, "size_z": spacing * 0.9,
                                 "material": mat["name"],
                                 "transform": _cols((1, 0, 0), (0, 1, 0), (0, 0, 1), (cx, 0.0, cz))}})
    sc = large_scene(width=width, height=height, max_depth=max_depth, dimension=dimension, sampler=sampler)
    sc["shapes"] = shapes
    sc["materials"] = materials
    sc["camera"]["param"]["transform"] = {"type": "look_at", "param": {
        "position": [0.0, 12.0, 30.0], "target_pos": [0.0, 0.0, 0.0], "up": [0.0, 1.0, 0.0]}}
    return sc
