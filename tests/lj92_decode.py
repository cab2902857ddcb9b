"""A minimal lossless JPEG (process 14, predictor 1) decoder for the streams
the DNG export writes, after the reference's own test decoder
(examples/prr2dng/lj92.rs:283-370): test infrastructure only."""


def decode(data: bytes):
    """(samples, width, height, components) of one stream; width is the JPEG
    width (samples per row / components)."""

    def be16(at):
        return data[at] << 8 | data[at + 1]

    at = 2
    width = height = components = 0
    table = {}
    while True:
        marker = data[at + 1]
        length = be16(at + 2)
        body = at + 4
        if marker == 0xC3:
            assert data[body] == 16
            height = be16(body + 1)
            width = be16(body + 3)
            components = data[body + 5]
        elif marker == 0xC4:
            counts = data[body + 1:body + 17]
            values = iter(data[body + 17:])
            code = 0
            for i, n in enumerate(counts):
                for _ in range(n):
                    table[(code, i + 1)] = next(values)
                    code += 1
                code <<= 1
        elif marker == 0xDA:
            at = body + length - 2
            break
        else:
            raise ValueError(f"unexpected marker {marker:x}")
        at = body + length - 2
    # Unstuff the entropy-coded segment up to EOI.
    raw = bytearray()
    while not (data[at] == 0xFF and data[at + 1] == 0xD9):
        raw.append(data[at])
        at += 2 if data[at] == 0xFF else 1
    bits = int.from_bytes(raw, "big") if raw else 0
    nbits = 8 * len(raw)
    pos = 0

    def take(n):
        nonlocal pos
        v = (bits >> (nbits - pos - n)) & ((1 << n) - 1)
        pos += n
        return v

    full_width = width * components
    out = []
    for i in range(full_width * height):
        code = length = 0
        while True:
            code = code << 1 | take(1)
            length += 1
            if (code, length) in table:
                ssss = table[(code, length)]
                break
            assert length < 16, "no code"
        if ssss == 0:
            d = 0
        elif ssss == 16:
            d = 32768
        else:
            v = take(ssss)
            d = v - (1 << ssss) + 1 if v < 1 << (ssss - 1) else v
        row, column = divmod(i, full_width)
        if column >= components:
            pred = out[i - components]
        elif row > 0:
            pred = out[i - full_width]
        else:
            pred = 1 << 15
        out.append((pred + d) & 0xFFFF)
    return out, width, height, components
