// DataStream control blocks on the host: which bytes of a datastream's
// receive ring hold a subintegration, the time of its first byte, and which
// of its FFTs have data.
//
// Restates DataStream::calculateControlParams (mpifxcorr/src/datastream.cpp:
// 376-636) and the VDIF frame alignment of VDIFDataStream::
// calculateControlParams (vdiffile.cpp:358-485), with the segment constants
// of DataStream::updateConfig and VDIFDataStream::updateConfig
// (datastream.cpp:741-787, vdiffile.cpp:490-505) and the subint byte count of
// Configuration::getDataBytes (configuration.cpp:807-842), for one
// configuration of real-sampled single-thread VDIF.  The
// decisions are integers computed from mixed int / long long / double
// expressions, so every expression keeps the reference's types and order.
// The ring's locking, MPI sends and reader threads are the caller's.

#include <cmath>
#include <cstdint>

#include "fxb_internal.h"

namespace fxb {

namespace {

const double kTiny = (double)0.000000001f;        // Mode::TINY is a float (mode.cpp:37)

long long gcd_ll(long long a, long long b)
{
	while(b != 0)
	{
		const long long r = a % b;
		a = b;
		b = r;
	}
	return a;
}

// Per-station constants of the ring's segments.
struct Seg {
	int numchannels, blockspersend, bpsnum, bpsden;
	int payloadbytes, framebytes, framespersecond, granularity;
	int sendbytes, nsinc, bytesbetweenintegerns;
	double sampletimens;
};

Seg segment_constants(const Job &job, int s, int readbytes, int guardns)
{
	const Job::Station &st = job.stations[s];
	const fxb_freq &f = job.freqs[st.band_freq[0]];
	Seg c;
	c.numchannels = f.nchan;
	c.blockspersend = job.blockspersend;
	// bytes per sample (configuration.cpp:1694-1702)
	c.bpsnum = (st.nband * st.nbits * 1) / 8;
	if(c.bpsnum == 0)
	{
		c.bpsnum = 1;
		c.bpsden = 8 / (st.nband * st.nbits * 1);
	}
	else
		c.bpsden = 1;
	c.sampletimens = 500.0 / f.bw_mhz;
	// bytes until the sample time is a whole number of ns again
	c.bytesbetweenintegerns = 0;
	double nsaccumulate = 0.0;
	do
	{
		nsaccumulate += c.bpsden * c.sampletimens;
		c.bytesbetweenintegerns += c.bpsnum;
	} while(!(std::fabs(nsaccumulate - int(nsaccumulate + 0.5)) < kTiny));
	c.payloadbytes = st.payload;
	c.framebytes = st.payload + st.header;
	// Configuration::getFramesPerSecond (configuration.cpp:667-681), stored as an int
	c.framespersecond = (int)(2.0e6 * f.bw_mhz * st.nband * st.nbits * 1 / (8 * st.payload));
	c.granularity = (int)(c.framespersecond / gcd_ll(c.framespersecond, 1000000000LL));
	// one subint's bytes: whole frames covering the subint and its guard,
	// with two frames of margin (Configuration::getDataBytes), stretched by
	// the guard (DataStream::updateConfig) and shrunk back to the subint
	// (VDIFDataStream::updateConfig)
	const int subintns = (int)job.subint_ns;
	int validlength = (1 * c.blockspersend * st.nband * 2 * st.nbits * c.numchannels) / 8;
	validlength += (1 * (int)(guardns / (1000.0 / (f.bw_mhz * 2.0)) + 1.0) * st.nband * st.nbits) / 8;
	const int numframes = validlength / c.payloadbytes + 2;
	const int databytes = numframes * c.framebytes;
	c.sendbytes = int((((long long)databytes) * ((long long)(subintns + guardns))) / subintns);
	c.sendbytes = int(((((double)c.sendbytes) * ((double)subintns)) / (subintns + guardns) + 0.5));
	// time span of one segment: its whole frames (VDIFDataStream::updateConfig)
	c.nsinc = int((readbytes / c.framebytes) * (1000000000.0 / double(c.framespersecond)) + 0.5);
	return c;
}

// Model::calculateDelayInterpolator at order 0 (model.cpp:229-269).
bool delay_order0(const DevStation &S, double offsettime, double *delay)
{
	if(S.npoly <= 0)
		return false;
	const double polyoffset = -S.poly0;
	int scansample = (int)((offsettime + polyoffset) / (double)S.interval);
	if(scansample == S.npoly && ((offsettime + polyoffset - scansample * S.interval) < 1e-6))
		scansample--;
	if(scansample < 0 || scansample >= S.npoly)
		return false;
	const double deltat = offsettime + polyoffset + 0.0 / 2.0 - scansample * S.interval;
	const double *cf = S.coeffs + scansample * (S.order + 1);
	double tp = 1.0, sum = 0.0;
	for(int i = 0; i <= S.order; i++)
	{
		sum += tp * cf[i];
		tp = tp * deltat;
	}
	*delay = sum;
	return true;
}

struct Out {
	int ctl1 = FXB_INVALID_SUBINT, ctl2 = 0;
	std::vector<int32_t> flags;
	bool pending = false;         // the ring does not reach the subint yet
};

// DataStream::calculateControlParams: the byte index of the subint's data in
// the ring, assuming no framing overhead, and the control words.
int base_control(const Seg &c, fxb_ring &ring, int scan, int offsetsec, int offsetns, double delayus1, double delayus2,
                 bool foundok, Out &o)
{
	const fxb_segment *seg = ring.seg;
	const int nseg = ring.nseg, readbytes = ring.readbytes;
	const long long bufferbytes = (long long)nseg * readbytes;
	int &at = ring.atsegment;
	const int bps = c.blockspersend;
	long long firstoffsetns = ((long long)offsetns) - static_cast<long long>(delayus1 * 1000);
	const int64_t dataspanns = static_cast<int64_t>(c.numchannels * c.blockspersend * 2 * c.sampletimens + 0.5);
	if(!foundok)
		return 0;
	long long lastoffsetns = (long long)offsetns + (long long)dataspanns + static_cast<long long>(-1000 * delayus2 + 0.5);
	for(int k = 0; k < 2; k++)
		if(lastoffsetns < 0)
		{
			offsetsec -= 1;
			firstoffsetns += 1000000000LL;
			lastoffsetns += 1000000000LL;
		}
	if(scan < seg[at].scan)
		return 0;
	if(!seg[at].readto)
		return 0;
	if(scan == seg[at].scan && offsetsec < seg[at].sec - 3)
		return 0;
	long long nsdifference = (offsetsec - seg[at].sec) * 1000000000LL + firstoffsetns - static_cast<long long>(seg[at].ns);
	long long validns = (static_cast<long long>(seg[at].validbytes) * static_cast<long long>(c.nsinc)) / readbytes;
	int laps = 0;
	while((scan > seg[at].scan || (scan == seg[at].scan && nsdifference >= validns)) &&
	      (ring.keepreading || (at != ring.lastvalid)))
	{
		// the datastream's main thread waits here for its reader; a ring that
		// comes round to where it started holds nothing newer yet
		if(++laps > nseg)
		{
			o.pending = true;
			return 0;
		}
		at = (at + 1) % nseg;
		nsdifference = (offsetsec - seg[at].sec) * 1000000000LL + firstoffsetns - static_cast<long long>(seg[at].ns);
		validns = (static_cast<long long>(seg[at].validbytes) * static_cast<long long>(c.nsinc)) / readbytes;
	}
	if((scan < seg[at].scan) || nsdifference < -c.nsinc)
		return 0;
	if(scan > seg[at].scan)
		return 0;
	const fxb_segment &cur = seg[at], &nxt = seg[(at + 1) % nseg];
	const int fftchannels = c.numchannels * 2;
	const int blockbytes = (fftchannels * c.bpsnum) / c.bpsden;
	const double currentsegmenttime = cur.sec + cur.ns / 1.0e9;
	const double nextsegmenttime = nxt.sec + nxt.ns / 1.0e9;
	const long long segstart = (long long)at * readbytes;
	if(cur.validbytes < readbytes || nxt.sec - cur.sec > 2 || nextsegmenttime < currentsegmenttime)
	{
		const double dbufferindex = segstart + ((((offsetsec - cur.sec) * 1.0e9 +
		                                          (firstoffsetns - static_cast<long long>(cur.ns))) / c.sampletimens) *
		                                        c.bpsnum) / c.bpsden;
		const int segoffbytes = int(dbufferindex - segstart);
		if(nextsegmenttime < currentsegmenttime && segoffbytes > cur.validbytes)
			return 0;
		if(dbufferindex < -blockbytes * c.blockspersend || dbufferindex > bufferbytes)
			return 0;
	}
	o.flags.assign(bps / kFlagsPerInt + 1, 0);
	o.ctl1 = cur.sec;
	long long bufferindex = segstart + (int(((offsetsec - cur.sec) * 1000000000LL +
	                                         (firstoffsetns - static_cast<long long>(cur.ns))) / c.sampletimens + 0.5) *
	                                    c.bpsnum) / c.bpsden;
	if(bufferindex % 2 != 0)
		bufferindex--;
	const long long gapns = (nxt.sec - cur.sec) * 1000000000LL + static_cast<long long>(nxt.ns) - static_cast<long long>(cur.ns);
	if(bufferindex == bufferbytes)
		if(cur.scan != nxt.scan || gapns - static_cast<long long>(c.nsinc) != 0)
		{
			o.ctl1 = FXB_INVALID_SUBINT;
			return 0;
		}
	int count = 0;
	while(bufferindex < segstart && count < bps)
	{
		bufferindex += blockbytes;
		count++;
	}
	if(bufferindex < segstart)
	{
		o.ctl1 = FXB_INVALID_SUBINT;
		return 0;
	}
	if(count > 0)
	{
		// the geometric delay changes over the skipped FFTs
		int tosubtract = (int(count * 1000.0 * (delayus2 - delayus1) / (c.sampletimens * bps) + 0.5) * c.bpsnum) / c.bpsden;
		if(bufferindex - tosubtract < segstart)
		{
			count++;
			bufferindex += blockbytes;
			if(count == bps)
			{
				o.ctl1 = FXB_INVALID_SUBINT;
				return 0;
			}
			tosubtract = (int(count * 1000.0 * (delayus2 - delayus1) / (c.sampletimens * bps) + 0.5) * c.bpsnum) / c.bpsden;
			bufferindex -= tosubtract;
		}
		bufferindex -= bufferindex % 2;
	}
	// back to a byte whose time is a whole number of ns
	int segoffbytes = (int)(bufferindex - segstart);
	bufferindex -= segoffbytes % c.bytesbetweenintegerns;
	segoffbytes -= segoffbytes % c.bytesbetweenintegerns;
	const long long segoffns =
	    static_cast<long long>(double(segoffbytes * c.bpsden / c.bpsnum) * c.sampletimens + 0.5);
	long long a = static_cast<long long>(o.ctl1) + (long long)segoffns / 1000000000LL;
	long long b = static_cast<long long>(cur.ns) + (long long)segoffns % 1000000000LL;
	a += b / 1000000000LL;
	b %= 1000000000LL;
	o.ctl1 = (int)a;
	o.ctl2 = (int)b;
	const bool nextcontinues = cur.validbytes == readbytes && gapns == c.nsinc;
	if((cur.validbytes - segoffbytes >= c.sendbytes) ||
	   (nextcontinues && (cur.validbytes - segoffbytes + nxt.validbytes) > c.sendbytes))
	{
		for(int i = count; i < bps; i++)
			o.flags[i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
	}
	else
	{
		const double dbufferindex = segstart + ((((offsetsec - cur.sec) * 1.0e9 +
		                                          (firstoffsetns - static_cast<long long>(cur.ns))) / c.sampletimens) *
		                                        c.bpsnum) / c.bpsden;
		if(dbufferindex < -blockbytes * c.blockspersend || dbufferindex > bufferbytes)
		{
			o.ctl1 = FXB_INVALID_SUBINT;
			return 0;
		}
		for(int i = count; i < bps; i++)
		{
			if(bufferindex + (long long)i * blockbytes - segstart < cur.validbytes)
				o.flags[i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
			else if(nextcontinues && (cur.validbytes - segoffbytes + nxt.validbytes) > (long long)i * blockbytes)
				o.flags[i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
		}
		// only the whole flag words are looked at (datastream.cpp:620-624)
		bool somegooddata = false;
		for(int i = 0; i < bps / kFlagsPerInt; i++)
			if(o.flags[i] > 0)
				somegooddata = true;
		if(!somegooddata)
		{
			o.ctl1 = FXB_INVALID_SUBINT;
			return 0;
		}
	}
	return (int)bufferindex;
}

}  // namespace

fxb_status datastream_control(const Job &job, const DevStation &S, int s, fxb_ring *ring, int scan, int sec, int ns,
                              const double *delay_us, int64_t *offset, int32_t *nbytes, int32_t *datasec,
                              int32_t *datans, int32_t *validflags, size_t nflagint, std::string &err)
{
	if(!ring || !ring->seg || ring->nseg < 1 || ring->readbytes <= 0 || ring->atsegment < 0 ||
	   ring->atsegment >= ring->nseg || !offset || !nbytes || !datasec || !datans)
	{
		err = "bad ring or output pointers";
		return FXB_ERR_ARG;
	}
	if(ring->guard_ns < 0 || job.subint_ns + ring->guard_ns > 2000000000LL)
	{
		err = "bad guard time";
		return FXB_ERR_ARG;
	}
	const Seg c = segment_constants(job, s, ring->readbytes, ring->guard_ns);
	const size_t nflags = (size_t)(c.blockspersend / kFlagsPerInt + 1);
	if(ring->readbytes % c.framebytes)
	{
		err = "ring segments must hold whole frames";
		return FXB_ERR_ARG;
	}
	if(validflags && nflagint < nflags)
	{
		err = "valid-flag buffer too small";
		return FXB_ERR_ARG;
	}
	// delays at the subint's start and end (datastream.cpp:389-396)
	double d1 = 0.0, d2 = 0.0;
	bool foundok = true;
	const int64_t dataspanns = static_cast<int64_t>(c.numchannels * c.blockspersend * 2 * c.sampletimens + 0.5);
	if(delay_us)
	{
		d1 = delay_us[0];
		d2 = delay_us[1];
	}
	else
	{
		foundok = delay_order0(S, (double)sec + ((double)ns) / 1.0e9, &d1);
		foundok = foundok && delay_order0(S, (double)sec + ((double)ns + dataspanns) / 1.0e9, &d2);
	}
	Out o;
	const int at0 = ring->atsegment;
	int bufferindex = base_control(c, *ring, scan, sec, ns, d1, d2, foundok, o);
	if(o.pending)
	{
		ring->atsegment = at0;
		err = "the ring's segments do not reach the subint yet: read further and ask again";
		return FXB_ERR_STATE;
	}
	if(o.ctl1 != FXB_INVALID_SUBINT)
	{
		// VDIF: back to the frame holding the byte, counted in payload bytes,
		// at the frame granularity; its time from the frame count
		const fxb_segment &cur = ring->seg[ring->atsegment];
		const long long bufferbytes = (long long)ring->nseg * ring->readbytes;
		const int vlbaoffset = bufferindex - ring->atsegment * ring->readbytes;
		if(vlbaoffset < 0)
			o.ctl1 = FXB_INVALID_SUBINT;
		else
		{
			int framesin = vlbaoffset / c.payloadbytes;
			if(framesin % c.granularity != 0)
				framesin -= (framesin % c.granularity);
			const long long segoffns = cur.ns + (long long)((1000000000.0 * framesin) / c.framespersecond);
			o.ctl1 = cur.sec + ((int)(segoffns / 1000000000));
			o.ctl2 = ((int)(segoffns % 1000000000));
			bufferindex = ring->atsegment * ring->readbytes + framesin * c.framebytes;
			if(bufferindex == bufferbytes)
			{
				const fxb_segment &nxt = ring->seg[(ring->atsegment + 1) % ring->nseg];
				// an int expression in the reference (vdiffile.cpp:466-468)
				const int32_t gap = (int32_t)((uint32_t)(nxt.sec - cur.sec) * 1000000000u + (uint32_t)nxt.ns -
				                              (uint32_t)cur.ns - (uint32_t)c.nsinc);
				if(cur.scan != nxt.scan || gap != 0)
					o.ctl1 = FXB_INVALID_SUBINT;
			}
			if(bufferindex > bufferbytes)
				o.ctl1 = FXB_INVALID_SUBINT;
		}
		if(o.ctl1 == FXB_INVALID_SUBINT)
			bufferindex = 0;
	}
	else
		bufferindex = 0;
	*offset = bufferindex;
	*nbytes = o.ctl1 == FXB_INVALID_SUBINT ? 0 : c.sendbytes;
	*datasec = o.ctl1;
	*datans = o.ctl1 == FXB_INVALID_SUBINT ? 0 : o.ctl2;
	if(validflags)
		for(size_t i = 0; i < nflags; i++)
			validflags[i] = i < o.flags.size() && o.ctl1 != FXB_INVALID_SUBINT ? o.flags[i] : 0;
	return FXB_OK;
}

}  // namespace fxb
