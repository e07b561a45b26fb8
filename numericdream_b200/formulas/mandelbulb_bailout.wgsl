// Mandelbulb whose escape radius is a parameter.  The built-in formula
// (src/gpu/shaders/mandelbrot.wgsl) steps with bulb_power_step, whose escape radius
// is the shader constant BULB_BAILOUT = 2 (template.wgsl:1013); the differentiation
// workload needs the radius as an input, so this file states the same power step
// with the comparison against p[2].  At Bailout = 2 it gives the built-in's DE.
// @param Power min=2 max=16 default=8
// @param Iterations min=2 max=16 default=12 int
// @param Bailout min=1 max=8 default=2
fn de_iterations(p: Params) -> i32 {
    return i32(p[1]);
}

fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> IterCarry {
    let power = p[0];
    let r = length(carry.z);
    if (r > p[2]) {
        return carry;
    }
    // spherical coordinates: polar angle from +z, azimuth atan2(y, x)
    let polar = acos(clamp(carry.z.z / r, -1.0, 1.0)) * power;
    let azim = atan2(carry.z.y, carry.z.x) * power;
    let r_pm1 = pow(r, power - 1.0);
    let s = sin(polar);
    let dir = vec3f(s * cos(azim), s * sin(azim), cos(polar));
    return IterCarry(r_pm1 * r * dir + pos, r_pm1 * power * carry.dr + 1.0);
}

fn de_finalize(carry: IterCarry) -> f32 {
    return bulb_log_escape(carry);
}
