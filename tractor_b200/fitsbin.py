"""Minimal FITS reading and writing (numpy only), enough for PsfEx model
files and Image.toFits / readFromFits: header cards of every HDU, binary
tables whose columns are fixed-size numeric arrays (TFORM letters L, B, I,
J, K, E, D; TDIM honoured), and image HDUs.  No compression, no
variable-length arrays, no scaling.  (The reference uses fitsio /
astrometry.util.fits.)
"""
import numpy as np

BLOCK = 2880
_TYPES = {'L': '?', 'B': 'u1', 'I': '>i2', 'J': '>i4', 'K': '>i8', 'E': '>f4', 'D': '>f8'}


def _parse_value(v):
    v = v.strip()
    if v.startswith("'"):
        end = v.find("'", 1)
        while end != -1 and end + 1 < len(v) and v[end + 1] == "'":   # escaped quote
            end = v.find("'", end + 2)
        return v[1:end].replace("''", "'").rstrip()
    v = v.split('/')[0].strip()
    if v in ('T', 'F'):
        return v == 'T'
    try:
        return int(v)
    except ValueError:
        pass
    try:
        return float(v.replace('D', 'E'))
    except ValueError:
        return v


def _read_header(data, off):
    """(ordered dict of keyword -> value, offset after the header)."""
    hdr = {}
    while True:
        if off + BLOCK > len(data):
            raise ValueError('truncated FITS header')
        block = data[off:off + BLOCK]
        off += BLOCK
        for i in range(BLOCK // 80):
            card = block[80 * i:80 * i + 80].decode('ascii', 'replace')
            key = card[:8].strip()
            if key == 'END':
                return hdr, off
            if card[8:10] == '= ':
                hdr[key] = _parse_value(card[10:])


def _data_bytes(hdr):
    naxis = int(hdr.get('NAXIS', 0))
    if naxis == 0:
        return 0
    n = abs(int(hdr['BITPIX'])) // 8
    for a in range(1, naxis + 1):
        n *= int(hdr['NAXIS%d' % a])
    return n + int(hdr.get('PCOUNT', 0))


def read_hdus(fn):
    """Every HDU of a FITS file as (header dict, data bytes)."""
    with open(fn, 'rb') as f:
        data = f.read()
    out, off = [], 0
    while off < len(data):
        if not data[off:off + 80].strip():
            break
        hdr, off = _read_header(data, off)
        n = _data_bytes(hdr)
        out.append((hdr, data[off:off + n]))
        off += (n + BLOCK - 1) // BLOCK * BLOCK
    return out


def _column_dtype(tform, tdim):
    tform = tform.strip()
    i = 0
    while i < len(tform) and tform[i].isdigit():
        i += 1
    count = int(tform[:i]) if i else 1
    code = tform[i:i + 1]
    if code not in _TYPES:
        raise ValueError('unsupported FITS column format %r' % tform)
    shape = (count,)
    if tdim:
        dims = [int(d) for d in tdim.strip().strip('()').split(',')]
        if int(np.prod(dims)) != count:
            raise ValueError('TDIM %r does not match TFORM %r' % (tdim, tform))
        shape = tuple(reversed(dims))   # FITS order is fastest-first
    return np.dtype((_TYPES[code], shape)) if shape != (1,) else np.dtype(_TYPES[code])


def read_table(fn, ext=1):
    """(header, {column name (lower case): numpy array (rows, ...)}) of the
    binary table in extension `ext`."""
    hdus = read_hdus(fn)
    if ext >= len(hdus):
        raise ValueError('%s has no extension %d' % (fn, ext))
    hdr, raw = hdus[ext]
    if hdr.get('XTENSION') != 'BINTABLE':
        raise ValueError('extension %d of %s is not a binary table' % (ext, fn))
    nrow, rowbytes = int(hdr['NAXIS2']), int(hdr['NAXIS1'])
    fields = []
    for c in range(1, int(hdr['TFIELDS']) + 1):
        fields.append((str(hdr['TTYPE%d' % c]).lower(),
                       _column_dtype(hdr['TFORM%d' % c], hdr.get('TDIM%d' % c))))
    dt = np.dtype(fields)
    if dt.itemsize != rowbytes:
        raise ValueError('row size %d does not match NAXIS1 %d' % (dt.itemsize, rowbytes))
    rec = np.frombuffer(raw[:nrow * rowbytes], dtype=dt, count=nrow)
    return hdr, {name: rec[name].astype(rec[name].dtype.newbyteorder('=')) for name, _ in fields}


def _card(key, value):
    if isinstance(value, bool):
        v = '%20s' % ('T' if value else 'F')
    elif isinstance(value, (int, np.integer)):
        v = '%20d' % value
    elif isinstance(value, (float, np.floating)):
        v = '%20s' % repr(float(value)).upper()
    else:
        v = "'%-8s'" % str(value).replace("'", "''")
    card = '%-8s= %s' % (key, v)
    if len(card) > 80:
        raise ValueError('FITS card too long: %s' % key)
    return card.ljust(80)


def _header_bytes(cards):
    txt = ''.join(cards) + 'END'.ljust(80)
    n = (len(txt) + BLOCK - 1) // BLOCK * BLOCK
    return txt.ljust(n).encode('ascii')


def write_table(fn, columns, header=None):
    """Writes a FITS file: an empty primary HDU and one binary table with
    the given columns ({name: array (rows, ...)}, float32 / float64 / int
    types) and extra header keywords (dict, in order)."""
    names = list(columns)
    nrow = len(columns[names[0]]) if names else 0
    fields, cards = [], []
    codes = {np.dtype('float32'): 'E', np.dtype('float64'): 'D', np.dtype('int16'): 'I',
             np.dtype('int32'): 'J', np.dtype('int64'): 'K', np.dtype('uint8'): 'B'}
    for c, name in enumerate(names, 1):
        a = np.asarray(columns[name])
        if len(a) != nrow:
            raise ValueError('columns must have the same number of rows')
        code = codes.get(a.dtype)
        if code is None:
            raise ValueError('unsupported column type %s' % a.dtype)
        shape = a.shape[1:]
        count = int(np.prod(shape)) if shape else 1
        fields.append((name.upper(), a.dtype.newbyteorder('>'), shape))
        cards += [_card('TTYPE%d' % c, name.upper()), _card('TFORM%d' % c, '%d%s' % (count, code))]
        if len(shape) > 1:
            cards.append(_card('TDIM%d' % c, '(%s)' % ','.join(str(d) for d in reversed(shape))))
    dt = np.dtype([(n, d, s) if s else (n, d) for n, d, s in fields])
    rec = np.zeros(nrow, dt)
    for name, (fname, _, _) in zip(names, fields):
        rec[fname] = columns[name]
    body = rec.tobytes()
    primary = [_card('SIMPLE', True), _card('BITPIX', 8), _card('NAXIS', 0),
               _card('EXTEND', True)]
    ext = [_card('XTENSION', 'BINTABLE'), _card('BITPIX', 8), _card('NAXIS', 2),
           _card('NAXIS1', dt.itemsize), _card('NAXIS2', nrow), _card('PCOUNT', 0),
           _card('GCOUNT', 1), _card('TFIELDS', len(names))] + cards
    for k, v in (header or {}).items():
        ext.append(_card(k, v))
    pad = (len(body) + BLOCK - 1) // BLOCK * BLOCK - len(body)
    with open(fn, 'wb') as f:
        f.write(_header_bytes(primary))
        f.write(_header_bytes(ext))
        f.write(body + b'\0' * pad)


# ---------------------------------------------------------------------------
# Image HDUs and a small file object with the calls Image.toFits /
# Image.readFromFits make on a fitsio.FITS (write, [i].read, [i].read_header)
# ---------------------------------------------------------------------------

_BITPIX = {np.dtype('uint8'): 8, np.dtype('int16'): 16, np.dtype('int32'): 32,
           np.dtype('int64'): 64, np.dtype('float32'): -32, np.dtype('float64'): -64}
_DTYPE = {8: 'u1', 16: '>i2', 32: '>i4', 64: '>i8', -32: '>f4', -64: '>f8'}


class FITSHDR(object):
    """An ordered FITS header: records of (name, value, comment)."""

    def __init__(self, records=None):
        self.records = []
        for r in records or []:
            self.add_record(r)

    def add_record(self, rec):
        name = str(rec['name']).upper()
        for r in self.records:
            if r['name'] == name:
                r['value'] = rec['value']
                r['comment'] = rec.get('comment', '')
                return
        self.records.append(dict(name=name, value=rec['value'], comment=rec.get('comment', '')))

    def __contains__(self, key):
        return any(r['name'] == str(key).upper() for r in self.records)

    def __getitem__(self, key):
        for r in self.records:
            if r['name'] == str(key).upper():
                return r['value']
        raise KeyError(key)

    def get(self, key, default=None):
        return self[key] if key in self else default

    def keys(self):
        return [r['name'] for r in self.records]


def _card_c(key, value, comment=''):
    card = _card(key, value)
    if comment:
        body = card.rstrip()
        room = 80 - len(body) - 3
        if room > 0:
            card = (body + ' / ' + comment[:room]).ljust(80)
    return card


class _HDU(object):
    def __init__(self, hdr, raw):
        self.hdr, self.raw = hdr, raw

    def read_header(self):
        return FITSHDR([dict(name=k, value=v) for k, v in self.hdr.items()])

    def read(self):
        naxis = int(self.hdr.get('NAXIS', 0))
        if naxis == 0:
            return None
        shape = tuple(int(self.hdr['NAXIS%d' % a]) for a in range(naxis, 0, -1))
        dt = np.dtype(_DTYPE[int(self.hdr['BITPIX'])])
        a = np.frombuffer(self.raw[:int(np.prod(shape)) * dt.itemsize], dtype=dt).reshape(shape)
        return a.astype(dt.newbyteorder('='))


class FITS(object):
    """A FITS file of image HDUs: write(data or None, header=...) appends an
    HDU (the first is the primary), fits[i].read() / .read_header() read
    them back.  mode 'rw' with clobber=True starts a new file."""

    def __init__(self, fn, mode='r', clobber=False):
        self.fn = fn
        self.hdus = []
        if mode == 'rw' and clobber:
            open(fn, 'wb').close()
        else:
            try:
                self.hdus = [_HDU(h, d) for h, d in read_hdus(fn)]
            except FileNotFoundError:
                if mode != 'rw':
                    raise
                open(fn, 'wb').close()

    def __len__(self):
        return len(self.hdus)

    def __getitem__(self, i):
        return self.hdus[i]

    def write(self, data, header=None):
        primary = len(self.hdus) == 0
        cards = []
        if data is None:
            arr = None
            cards += [_card('SIMPLE', True) if primary else _card('XTENSION', 'IMAGE'),
                      _card('BITPIX', 8), _card('NAXIS', 0)]
        else:
            arr = np.ascontiguousarray(data)
            if arr.dtype not in _BITPIX:
                arr = arr.astype(np.float64)
            cards += [_card('SIMPLE', True) if primary else _card('XTENSION', 'IMAGE'),
                      _card('BITPIX', _BITPIX[arr.dtype]), _card('NAXIS', arr.ndim)]
            cards += [_card('NAXIS%d' % (a + 1), arr.shape[arr.ndim - 1 - a])
                      for a in range(arr.ndim)]
        if primary:
            cards.append(_card('EXTEND', True))
        else:
            cards += [_card('PCOUNT', 0), _card('GCOUNT', 1)]
        for r in (header.records if isinstance(header, FITSHDR) else
                  [dict(name=k, value=v) for k, v in (header or {}).items()]):
            cards.append(_card_c(r['name'], r['value'], r.get('comment', '')))
        body = b'' if arr is None else arr.astype(arr.dtype.newbyteorder('>')).tobytes()
        pad = (len(body) + BLOCK - 1) // BLOCK * BLOCK - len(body)
        with open(self.fn, 'ab') as f:
            f.write(_header_bytes(cards))
            f.write(body + b'\0' * pad)
        self.hdus = [_HDU(h, d) for h, d in read_hdus(self.fn)]

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
